"""Batched ensembles: every member of an ensemble of uneven 2-D and 1-D runs
(one persistent sweep launch per direction for all members, one CUDA graph
per step) must equal the same run advanced alone through how_run, bit for
bit -- state, face B, time and step count -- whatever tile shapes the sweeps
use, and one member is checked against the CPU oracle."""
import numpy as np
import pytest

from howtest import CPUOracle, active, rel_l1

pytestmark = pytest.mark.gpu


def _members(hm):
    P = hm.make_parameters
    return [
        P(nx=32, ny=32, nz=1, nt=1, tend=0.05, gam=1.45, cour=0.4, problem="orszag_tang"),
        P(nx=64, ny=48, nz=1, nt=2, tend=0.04, gam=5.0 / 3.0, cour=0.4, problem="orszag_tang"),
        P(nx=48, ny=48, nz=1, nt=1, tend=0.01, gam=1.4, cour=0.4, problem="mhd_rotor",
          x1bc="open", x2bc="open", x3bc="periodic"),
        P(nx=200, ny=1, nz=1, nt=1, tend=0.03, gam=2.0, cour=0.4, problem="brio_wu",
          x1bc="open", x2bc="open", x3bc="open"),
        P(nx=96, ny=1, nz=1, nt=3, tend=0.02, gam=2.0, cour=0.4, problem="brio_wu",
          x1bc="open", x2bc="open", x3bc="open"),
        P(nx=16, ny=80, nz=1, nt=1, tend=0.02, gam=1.6, cour=0.4, problem="orszag_tang"),
    ]


def _alone(hm, p):
    with hm.Domain(p) as d:
        d.init_problem()
        t, s, _ = d.run(0.0, -1)
        return d.get_state(0), d.get_face_b(0), t, s


def _run_ensemble(hm, params, shapes=None, chunks=None):
    with hm.Ensemble(params) as e:
        e.init()
        if shapes is not None:
            e.set_shapes(*shapes)
        if chunks:
            for c in chunks:
                e.run(c)
        e.run(-1)
        out = []
        for m in range(len(params)):
            t, s, done = e.status(m)
            assert done
            d = e.members[m]
            out.append((d.get_state(0), d.get_face_b(0), t, s))
        return out, e.shapes()


@pytest.fixture(scope="module")
def alone():
    import how_mhd as hm
    return [_alone(hm, p) for p in _members(hm)]


def _same(a, b):
    np.testing.assert_array_equal(a[0], b[0])
    for x, y in zip(a[1], b[1]):
        np.testing.assert_array_equal(x, y)
    assert a[2] == b[2] and a[3] == b[3]


def test_ensemble_autotuned_equals_single_runs(alone):
    import how_mhd as hm
    out, (shapes, ms) = _run_ensemble(hm, _members(hm))
    for a, b in zip(out, alone):
        _same(a, b)
    assert all(0 <= s < 3 for s in shapes)
    assert (ms[0] > 0).all() and (ms[1] > 0).all()   # every candidate was timed


@pytest.mark.parametrize("shapes", [(0, 0, 0), (1, 1, 0), (2, 2, 0)])
def test_ensemble_every_shape_bitwise(alone, shapes):
    import how_mhd as hm
    out, _ = _run_ensemble(hm, _members(hm), shapes=shapes)
    for a, b in zip(out, alone):
        _same(a, b)


def test_ensemble_in_chunks_equals_single_runs(alone):
    import how_mhd as hm
    out, _ = _run_ensemble(hm, _members(hm), shapes=(1, 2, 0), chunks=[1, 5, 17])
    for a, b in zip(out, alone):
        _same(a, b)


def test_ensemble_member_vs_oracle():
    """A member against the CPU oracle under the parity suite's bar (relative
    L1 <= 1e-12 per conserved variable, Orszag-Tang 128^2, ~7 steps)."""
    import how_mhd as hm
    p = hm.make_parameters(nx=128, ny=128, nz=1, nt=1, tend=0.006, gam=5.0 / 3.0, cour=0.4,
                           problem="orszag_tang")
    bw = hm.make_parameters(nx=64, ny=1, nz=1, nt=1, tend=0.01, gam=2.0, cour=0.4, problem="brio_wu",
                            x1bc="open", x2bc="open", x3bc="open")
    with hm.Ensemble([p, bw]) as e:
        e.init()
        e.run(-1)
        q = e.members[0].get_state(0)
        t, steps, _ = e.status(0)
    o = CPUOracle(128, 128, 1, gam=5.0 / 3.0, rhomin=p.rhomin, pgmin=p.pgmin)
    o.init_problem("orszag_tang")
    rc, to, dts = o.run(0.006)
    assert rc == 0 and len(dts) == steps and steps <= 10
    err = rel_l1(active(q, 128, 128, 1), active(o.get_q(0), 128, 128, 1))
    assert np.all(err <= 1e-12), err


def test_ensemble_rejects_bad_members():
    import how_mhd as hm
    with pytest.raises(hm.HowError):
        hm.Ensemble([hm.make_parameters(nx=1, ny=16, nz=1, problem="orszag_tang")])
    with pytest.raises(hm.HowError):
        hm.Ensemble([hm.make_parameters(nx=16, ny=16, nz=1, problem="orszag_tang", precision="mixed")])
