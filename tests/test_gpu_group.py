"""A domain decomposed into z slabs (how_group) against the same run on the
whole domain (how_run): the parts run the whole-domain kernels and their
halos are exact plane copies, so state, face B and the dt sequence must be
equal bit for bit.  The parts share the one GPU here (one stream each); on a
node they sit on separate GPUs and the copies go peer to peer.

Covers the reference's MPI decomposition semantics: the q, face-B and CT
halo exchanges (src/bound.cpp:132-271, src/fluxct.cpp:287-479, 554-751), the
dt allreduce (src/tstep.cpp:87-121), periodic wrap-around between the first
and last part, and open z boundaries filled only on each part's physical side
(the reference fills both sides of a rank with one physical side,
src/bound.cpp:273-291)."""
import numpy as np
import pytest

from howtest import active

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prob,n,bc,nparts,steps", [
    ("blast3d_b", (24, 20, 32), ("periodic",) * 3, 2, 5),
    ("blast3d_b", (16, 16, 27), ("periodic",) * 3, 3, 3),
    ("mpi_smooth3d", (20, 16, 18), ("periodic", "open", "open"), 3, 4),
    ("mpi_smooth3d", (12, 10, 12), ("open", "periodic", "open"), 4, 3),
    ("alfven3d", (16, 16, 16), ("periodic",) * 3, 1, 3),
], ids=["blast_2parts", "blast_3parts_uneven", "smooth_3parts_open_z", "smooth_4parts_open_xz", "alfven_1part"])
def test_group_equals_whole_domain(prob, n, bc, nparts, steps):
    import how_mhd as hm
    p = hm.make_parameters(nx=n[0], ny=n[1], nz=n[2], nt=1, tend=10.0, gam=5.0 / 3.0, cour=0.4, problem=prob,
                           x1bc=bc[0], x2bc=bc[1], x3bc=bc[2], rhomin=1e-6, pgmin=1e-6)
    with hm.Domain(p) as dom:
        dom.init_problem()
        t, s, dts = dom.run(0.0, steps, dts_cap=steps)
        q = active(dom.get_state(0), *n)
        b = [active(x, *n) for x in dom.get_face_b(0)]
    with hm.Group(p, nparts) as g:
        ranges = [g.part_range(k) for k in range(nparts)]
        assert ranges[0][0] == 0 and sum(r[1] for r in ranges) == n[2]
        g.init_problem()
        tg, sg, dtg = g.run(0.0, steps, dts_cap=steps)
        qg = active(g.get_state(), *n)
        bg = [active(x, *n) for x in g.get_face_b()]
    assert sg == s == steps and tg == t
    np.testing.assert_array_equal(dtg, dts)
    np.testing.assert_array_equal(qg, q)
    for c in range(3):
        np.testing.assert_array_equal(bg[c], b[c])


def test_group_rejects_thin_parts():
    import how_mhd as hm
    p = hm.make_parameters(nx=8, ny=8, nz=8, nt=1, tend=1.0, problem="uniform")
    with pytest.raises(hm.HowError) as e:
        hm.Group(p, 3)
    assert e.value.code == -1 and "3 z planes per part" in str(e.value)
