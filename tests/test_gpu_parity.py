"""Parity of the B200 path (through the C ABI) with the CPU oracle.

Bar (FP64 path): relative L1 per conserved variable <= 1e-12 after 10 steps,
dt identical to 1e-14 relative, face B to 1e-12.  Comparisons use active cells
only: the reference leaves collapsed-axis ghost planes stale (2-D/1-D) and its
ghost cells are refilled every stage."""
import numpy as np
import pytest

from howtest import CPUOracle, active, rel_l1

pytestmark = pytest.mark.gpu

TOL_Q = 1e-12
# dt of the fast FP64 path: the reference's own dt moves by up to 4.7e-14
# (Orszag-Tang, 10 steps) when its initial state is perturbed by 1e-16, so a
# path that rounds differently cannot be held to 1e-14; 1e-13 is ~2x that
# self-sensitivity.  The bit-reproducing mode is held to 0.
TOL_DT = 1e-13


def _hm():
    import how_mhd as hm
    return hm


def _setup(prob, n, bc, gam, tend=1.0, **extra):
    hm = _hm()
    kw = dict(nx=n[0], ny=n[1], nz=n[2], nt=1, tend=tend, gam=gam, cour=0.4, problem=prob,
              x1bc=bc[0], x2bc=bc[1], x3bc=bc[2])
    kw.update(extra)
    p = hm.make_parameters(**kw)
    dom = hm.Domain(p)
    o = CPUOracle(*n, bc=bc, gam=gam, rhomin=p.rhomin, pgmin=p.pgmin,
                  size=(p.xsize, p.ysize, p.zsize))
    return hm, p, dom, o


def _perturbed_state(hm, p, seed, amp=0.02):
    """A problem state with seeded smooth-ish noise on every variable (active cells)."""
    q = hm.problem_state(p)
    rng = np.random.default_rng(seed)
    a = active(q, p.nx, p.ny, p.nz)
    a *= 1.0 + amp * rng.standard_normal(a.shape)
    return q


# Well-conditioned configurations: the reference's own result moves by less
# than ~1e-13 under 1e-16 input noise.
CASES = [
    # name, problem, n, bc, gam, steps
    ("ot128", "orszag_tang", (128, 128, 1), ("periodic",) * 3, 5.0 / 3.0, 10),
    ("blastb32", "blast3d_b", (32, 32, 32), ("periodic",) * 3, 5.0 / 3.0, 10),
    ("smooth_mixed", "mpi_smooth3d", (20, 14, 12), ("periodic", "open", "periodic"), 5.0 / 3.0, 6),
    ("alfven24", "alfven3d", (24, 24, 24), ("periodic",) * 3, 5.0 / 3.0, 6),
]

# Ill-conditioned configurations: B parallel to a sweep axis (blast3d, rotor)
# or a mean transverse B of exactly zero (Brio-Wu's discontinuity) send the
# reference into its degenerate-eigenvector branch (src/ssprk.cpp:641-647),
# whose basis is picked by round-off noise.  The reference itself moves by
# 5.6e-4 / 3.1e-7 / 1.7e-11 (relative L1 after 10 steps) under 1e-16 input
# noise; the fast FP64 path must stay within 10x that self-sensitivity, which
# the test measures with the oracle.
ILL = [
    ("blast32", "blast3d", (32, 32, 32), ("periodic",) * 3, 5.0 / 3.0, 10),
    ("rotor64_open", "mhd_rotor", (64, 64, 1), ("open", "open", "periodic"), 1.4, 10),
    ("briowu400", "brio_wu", (400, 1, 1), ("open",) * 3, 2.0, 10),
]


def _run_both(prob, n, bc, gam, steps, q_override=None):
    hm, p, dom, o = _setup(prob, n, bc, gam, tend=10.0)
    q0 = hm.problem_state(p) if q_override is None else q_override
    dom.set_state(q0)
    dom.bound(0)
    dom.initialize_bfield_from_q()
    o.set_state(q0)
    t, s, dts = dom.run(0.0, steps, dts_cap=steps)
    rc, to, odts = o.run(10.0, 1, steps)
    assert s == steps and len(odts) == steps
    return hm, p, dom, o, dts, odts


@pytest.mark.parametrize("name,prob,n,bc,gam,steps", CASES, ids=[c[0] for c in CASES])
def test_run_parity(name, prob, n, bc, gam, steps):
    hm, p, dom, o, dts, odts = _run_both(prob, n, bc, gam, steps)
    np.testing.assert_allclose(dts, odts, rtol=TOL_DT, atol=0)
    qg = active(dom.get_state(0), *n)
    qo = active(o.get_q(0), *n)
    err = rel_l1(qg, qo)
    assert np.all(err <= TOL_Q), f"{name}: rel L1 per var {err}"
    bg = dom.get_face_b(0)
    bo = o.get_faceb(0)
    for c in range(3):
        e = rel_l1(active(bg[c], *n)[None], active(bo[c], *n)[None])[0]
        assert e <= TOL_Q, f"{name}: face B{c} rel L1 {e}"


@pytest.mark.parametrize("name,prob,n,bc,gam,steps", ILL, ids=[c[0] for c in ILL])
def test_run_parity_ill_conditioned(name, prob, n, bc, gam, steps):
    hm, p, dom, o, dts, odts = _run_both(prob, n, bc, gam, steps)
    qg = active(dom.get_state(0), *n)
    qo = active(o.get_q(0), *n)
    err = rel_l1(qg, qo)
    # the oracle's own sensitivity: same run from a 1e-16-perturbed state
    q0 = hm.problem_state(p)
    rng = np.random.default_rng(0)
    a = active(q0, *n)
    a *= 1.0 + 1e-16 * rng.standard_normal(a.shape)
    o2 = CPUOracle(*n, bc=bc, gam=gam, rhomin=p.rhomin, pgmin=p.pgmin)
    o2.set_state(q0)
    o2.run(10.0, 1, steps)
    sens = rel_l1(active(o2.get_q(0), *n), qo)
    bound = 10.0 * np.maximum(sens, 1e-13)
    assert np.all(err <= bound), f"{name}: rel L1 {err} vs 10x self-sensitivity {bound}"


def test_bound_bitwise():
    hm, p, dom, o = _setup("mpi_smooth3d", (10, 7, 5), ("periodic", "open", "periodic"), 5.0 / 3.0)
    rng = np.random.default_rng(1)
    q = rng.standard_normal((8,) + p.shape)
    dom.set_state(q)
    dom.bound(0)
    o.set_state(q, faceb=[np.zeros(p.shape)] * 3)
    np.testing.assert_array_equal(dom.get_state(0), o.get_q(0))


def test_bound_collapsed_axis_bitwise():
    """n = 1 and n = 2 axes reproduce the reference's in-place fill order."""
    hm, p, dom, o = _setup("uniform", (6, 1, 2), ("periodic", "periodic", "open"), 5.0 / 3.0)
    rng = np.random.default_rng(2)
    q = rng.standard_normal((8,) + p.shape)
    dom.set_state(q)
    dom.bound(0)
    o.set_state(q, faceb=[np.zeros(p.shape)] * 3)
    np.testing.assert_array_equal(dom.get_state(0), o.get_q(0))


def test_init_faceb_and_tstep():
    hm, p, dom, o = _setup("mpi_smooth3d", (24, 20, 16), ("periodic",) * 3, 5.0 / 3.0)
    q = _perturbed_state(hm, p, 3)
    dom.set_state(q)
    dom.bound(0)
    dom.initialize_bfield_from_q()
    o.set_state(q)
    for c, (bg, bo) in enumerate(zip(dom.get_face_b(0), o.get_faceb(0))):
        np.testing.assert_allclose(active(bg, 24, 20, 16), active(bo, 24, 20, 16), rtol=1e-14, atol=1e-15)
    assert abs(dom.tstep() / o.tstep() - 1.0) <= TOL_DT


@pytest.mark.parametrize("direction", [0, 1, 2])
def test_single_sweep(direction):
    n = (36, 20, 18)
    hm, p, dom, o = _setup("mpi_smooth3d", n, ("periodic", "open", "periodic"), 5.0 / 3.0)
    q = _perturbed_state(hm, p, 10 + direction, amp=0.05)
    dom.set_state(q)
    dom.bound(0)
    dom.initialize_bfield_from_q()
    o.set_state(q)
    dt = 0.8 * o.tstep()
    q1o, ao, bo = o.sweep(direction, dt)
    dom.sweep(direction, dt)
    q1g = dom.get_state(1)
    err = rel_l1(active(q1g, *n), active(q1o, *n))
    assert np.all(err <= TOL_Q), f"sweep {direction}: {err}"
    ia, ib = [(0, 1), (3, 2), (4, 5)][direction]
    # CT faces: padded face index 2..n+2 along the sweep, active transverse
    sl = [slice(3, n[0] + 3), slice(3, n[1] + 3), slice(3, n[2] + 3)]
    sl[direction] = slice(2, n[direction] + 3)
    for w, ref in ((ia, ao), (ib, bo)):
        g = dom.get_ct_array(w)[tuple(sl)]
        r = ref[tuple(sl)]
        e = np.abs(g - r).sum() / max(np.abs(r).sum(), 1e-300)
        assert e <= TOL_Q, f"sweep {direction} CT array {w}: {e}"


def test_ct_avg4_vs_oracle():
    """The optional fourth-order CT face average (ct_avg 4) against the
    oracle run with the same option, 10 steps of the 3-D smooth wave."""
    from howtest import oracle_lib
    hm, p, dom, o = _setup("alfven3d", (24, 24, 24), ("periodic",) * 3, 5.0 / 3.0, ct_avg=4)
    lib = oracle_lib()
    lib.oracle_set_ct_avg(4)
    try:
        q0 = hm.problem_state(p)
        o.set_state(q0)
        rc, t_o, dts_o = o.run(1.0, max_steps=10)
        qo = o.get_q(0)
    finally:
        lib.oracle_set_ct_avg(2)
    with dom:
        dom.init_problem()
        t, s, dts = dom.run(0.0, 10, dts_cap=10)
        q = dom.get_state(0)
    np.testing.assert_allclose(dts, dts_o, rtol=1e-13)
    a, b = active(q, 24, 24, 24), active(qo, 24, 24, 24)
    for v in range(8):
        sc = np.abs(b[v]).sum()
        if sc > 0:
            assert np.abs(a[v] - b[v]).sum() <= 1e-12 * sc, v
