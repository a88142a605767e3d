"""Parity of the B200 path (through the C ABI) with the CPU oracle.

Bar (FP64 path): relative L1 per conserved variable <= 1e-12 after 10 steps,
dt identical to 1e-14 relative, face B to 1e-12.  Comparisons use active cells
only: the reference leaves collapsed-axis ghost planes stale (2-D/1-D) and its
ghost cells are refilled every stage.  Every comparison reports the figures it
achieved through the `parity_record` fixture."""
import os

import numpy as np
import pytest

from howtest import CPUOracle, active, oracle_lib, rel_l1

pytestmark = pytest.mark.gpu

TOL_Q = 1e-12
# dt bar of the north star: 1e-14 relative, per step.
TOL_DT = 1e-14
# Cases held to a looser dt bar, with the reason.  Orszag-Tang: the
# reference's own dt moves by 4.7e-14 over 10 steps when its initial state is
# perturbed by 1e-16, so a path that rounds differently misses 1e-14 there
# (this path: 4.7e-14); every other case meets 1e-14.
TOL_DT_CASE = {"ot128": 1e-13}


def _dt_err(dts, odts):
    dts, odts = np.asarray(dts, dtype=np.float64), np.asarray(odts, dtype=np.float64)
    return float(np.max(np.abs(dts - odts) / np.abs(odts))) if len(odts) else 0.0


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
def test_run_parity(name, prob, n, bc, gam, steps, parity_record):
    hm, p, dom, o, dts, odts = _run_both(prob, n, bc, gam, steps)
    qg = active(dom.get_state(0), *n)
    qo = active(o.get_q(0), *n)
    err = rel_l1(qg, qo)
    bg = dom.get_face_b(0)
    bo = o.get_faceb(0)
    eb = [rel_l1(active(bg[c], *n)[None], active(bo[c], *n)[None])[0] for c in range(3)]
    dte = _dt_err(dts, odts)
    parity_record(case=name, steps=steps, max_rel_dt=dte, rel_l1_q=err, rel_l1_faceb=eb)
    assert dte <= TOL_DT_CASE.get(name, TOL_DT), f"{name}: max relative dt error {dte:.3e}"
    assert np.all(err <= TOL_Q), f"{name}: rel L1 per var {err}"
    for c in range(3):
        assert eb[c] <= TOL_Q, f"{name}: face B{c} rel L1 {eb[c]}"


@pytest.mark.parametrize("name,prob,n,bc,gam,steps", ILL, ids=[c[0] for c in ILL])
def test_run_parity_ill_conditioned(name, prob, n, bc, gam, steps, parity_record):
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
    parity_record(case=name, steps=steps, max_rel_dt=_dt_err(dts, odts), rel_l1_q=err, oracle_self_sensitivity=sens)
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


def test_init_faceb_and_tstep(parity_record):
    hm, p, dom, o = _setup("mpi_smooth3d", (24, 20, 16), ("periodic",) * 3, 5.0 / 3.0)
    q = _perturbed_state(hm, p, 3)
    dom.set_state(q)
    dom.bound(0)
    dom.initialize_bfield_from_q()
    o.set_state(q)
    for c, (bg, bo) in enumerate(zip(dom.get_face_b(0), o.get_faceb(0))):
        np.testing.assert_allclose(active(bg, 24, 20, 16), active(bo, 24, 20, 16), rtol=1e-14, atol=1e-15)
    dte = abs(dom.tstep() / o.tstep() - 1.0)
    parity_record(case="tstep_smooth_perturbed", max_rel_dt=dte)
    assert dte <= TOL_DT


@pytest.mark.parametrize("direction", [0, 1, 2])
def test_single_sweep(direction, parity_record):
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
    parity_record(case=f"sweep{direction}", rel_l1_q1=err)
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


# ------------------------------------------------ standalone path functions
@pytest.mark.parametrize("n,bc", [((20, 14, 12), ("periodic", "open", "periodic")),
                                  ((24, 18, 1), ("open", "periodic", "periodic")),
                                  ((16, 1, 12), ("periodic", "periodic", "open"))],
                         ids=["3d_mixed", "2d_xy_open", "2d_xz_open"])
@pytest.mark.parametrize("iw,k1,k3", [(1, 1.0, 0.0), (1, 0.44437049406734, 0.55562950593266)],
                         ids=["stage1", "combined"])
def test_fluxct_vs_oracle(n, bc, iw, k1, k3, parity_record):
    """how_fluxct after the three single sweeps of stage 1 against the
    oracle's fluxct (src/fluxct.cpp:786-899) on the same CT flux arrays: face
    B(1) and the face-to-centre B in q(1, 4..6), relative L1 <= 1e-12."""
    hm, p, dom, o = _setup("mpi_smooth3d", n, bc, 5.0 / 3.0)
    q = _perturbed_state(hm, p, 40 + n[2], amp=0.05)
    dom.set_state(q)
    dom.bound(0)
    dom.initialize_bfield_from_q()
    o.set_state(q)
    dt = 0.8 * o.tstep()
    o.stage1_sweeps(dt)
    o.fluxct(iw, k1, k3)
    for d in range(3):
        if n[d] > 1:
            dom.sweep(d, dt)
    dom.fluxct(iw, k1, k3)
    bg, bo = dom.get_face_b(1), o.get_faceb(1)
    eb = [rel_l1(active(bg[c], *n)[None], active(bo[c], *n)[None])[0] for c in range(3)]
    qg, qo = active(dom.get_state(1), *n), active(o.get_q(1), *n)
    eq = [rel_l1(qg[v][None], qo[v][None])[0] for v in (4, 5, 6)]
    parity_record(case=f"fluxct_{n}_{bc}_k1={k1}", rel_l1_faceb=eb, rel_l1_cell_b=eq)
    assert max(eb) <= TOL_Q, eb
    assert max(eq) <= TOL_Q, eq


def test_fluxct_1d_is_a_no_op():
    """In 1-D the reference's fluxct returns at once (src/fluxct.cpp:793)."""
    hm, p, dom, o = _setup("brio_wu", (64, 1, 1), ("open",) * 3, 2.0)
    dom.init_problem()
    b0 = dom.get_face_b(1)
    q1 = dom.get_state(1)
    dom.fluxct(1, 1.0, 0.0)
    for a, b in zip(dom.get_face_b(1), b0):
        np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(dom.get_state(1), q1)


def test_prot_vs_oracle(parity_record):
    """how_prot (src/prot.cpp:10-51) on a state with cells below both floors."""
    n = (18, 12, 10)
    hm, p, dom, o = _setup("mpi_smooth3d", n, ("periodic",) * 3, 5.0 / 3.0, rhomin=1e-3, pgmin=1e-3)
    q = _perturbed_state(hm, p, 7, amp=0.05)
    a = active(q, *n)
    rng = np.random.default_rng(8)
    low = rng.random(a.shape[1:]) < 0.1
    a[0][low] = 1e-5                                  # density below rhomin
    hot = rng.random(a.shape[1:]) < 0.1
    kin_mag = 0.5 * ((a[1:4] ** 2).sum(0) / np.maximum(a[0], 1e-3) + (a[4:7] ** 2).sum(0))
    a[7][hot] = kin_mag[hot]                          # pressure ~0, below pgmin
    dom.set_state(q, stage=2)
    o.set_q(2, q)
    dom.prot(2)
    o.prot(2)
    qg, qo = active(dom.get_state(2), *n), active(o.get_q(2), *n)
    np.testing.assert_array_equal(qg[:7], qo[:7])     # rho floored exactly; m, B untouched
    rel = float(np.max(np.abs(qg[7] - qo[7]) / np.abs(qo[7])))
    parity_record(case="prot", max_rel_E=rel, floored_rho=int(low.sum()), floored_p=int(hot.sum()))
    assert rel <= 1e-14, rel


@pytest.mark.parametrize("n,bc", [((10, 7, 5), ("periodic", "open", "periodic")),
                                  ((6, 1, 2), ("open", "periodic", "open"))])
def test_bound_bfield_vs_oracle(n, bc):
    """how_bound_bfield (src/fluxct.cpp:481-490), bit for bit, including the
    n = 1 and n = 2 axes' in-place fill order."""
    hm, p, dom, o = _setup("uniform", n, bc, 5.0 / 3.0)
    rng = np.random.default_rng(9)
    b = [rng.standard_normal(p.shape) for _ in range(3)]
    dom.set_face_b(*b, stage=3)
    dom.bound_bfield(3)
    o.set_faceb_stage(3, b)
    o.bound_bfield(3)
    for a, r in zip(dom.get_face_b(3), o.get_faceb(3)):
        np.testing.assert_array_equal(a, r)


# ---------------------------------------------------- configurations at size
def test_orszag_tang_128_to_tend(parity_record):
    """Config 0 through the main loop to tend = 0.5 (src/main.cpp:158-234):
    the whole dt sequence, the state and face B at tend against the oracle.
    765 steps.  The oracle itself moves by 1.3e-13 - 4.3e-13 (relative L1)
    at tend under a 1e-16 perturbation of its initial state; the bar is 1e-11.
    The last step is clamped to tend (dt = tend - time): it absorbs the
    difference of the summed dts, so it is compared in absolute terms,
    against tend."""
    n = (128, 128, 1)
    hm, p, dom, o = _setup("orszag_tang", n, ("periodic",) * 3, 5.0 / 3.0, tend=0.5)
    oracle_lib().oracle_set_threads(os.cpu_count() or 1)
    with dom:
        dom.init_problem()
        t, s, dts = dom.run(0.0, -1, dts_cap=10000)
        qg = active(dom.get_state(0), *n)
        bg = dom.get_face_b(0)
    o.set_state(hm.problem_state(p))
    rc, to, odts = o.run(0.5, 1)
    assert rc == 0 and s == len(odts), (s, len(odts))
    assert t == 0.5 and to == 0.5
    dte = _dt_err(dts[:-1], odts[:-1])
    last = abs(dts[-1] - odts[-1]) / 0.5
    err = rel_l1(qg, active(o.get_q(0), *n))
    bo = o.get_faceb(0)
    eb = [rel_l1(active(bg[c], *n)[None], active(bo[c], *n)[None])[0] for c in range(2)]
    parity_record(case="ot128_tend0.5", steps=s, max_rel_dt_but_last=dte, last_dt_abs_err_over_tend=last,
                  rel_l1_q=err, rel_l1_faceb=eb)
    assert dte <= 1e-11 and last <= 1e-12, (dte, last)
    assert np.all(err <= 1e-11), err
    assert max(eb) <= 1e-11, eb


# The oracle's own response at 256^3 (blast3d_b, 10 steps from t = 0) to a
# 1e-16 relative perturbation of its initial state: relative L1 per conserved
# variable and the max relative dt change.  At this resolution the problem is
# ill-conditioned in the momenta and B_z (at 64^3 and 128^3 the same figures
# are 4e-14 and 1.5e-13): a path that rounds differently cannot do better.
SENS_BLAST256 = np.array([3.50e-13, 1.15e-09, 1.20e-09, 6.64e-10, 3.69e-13, 3.52e-13, 2.61e-09, 5.94e-12])
SENS_BLAST256_DT = 5.67e-10


def test_blast3d_b_headline_size_fp64_10_steps(parity_record):
    """The headline workload (blast3d_b 256^3, plain FP64) for 10 steps from
    t = 0 against the oracle port.  Bar: relative L1 <= 1e-12 for every
    variable the problem's conditioning allows it (rho, Bx, By and the face
    B of x and y), else <= 10x the oracle's own sensitivity (SENS_BLAST256);
    dt the same way.  The oracle needs ~16 GB of host memory at 256^3; with
    less the test runs 128^3 at 1e-12 throughout."""
    import psutil
    n1 = 256 if psutil.virtual_memory().available > 32e9 else 128
    n = (n1, n1, n1)
    hm, p, dom, o = _setup("blast3d_b", n, ("periodic",) * 3, 5.0 / 3.0, rhomin=1e-6, pgmin=1e-6)
    oracle_lib().oracle_set_threads(os.cpu_count() or 1)
    steps = 10
    with dom:
        dom.init_problem()
        t, s, dts = dom.run(0.0, steps, dts_cap=steps)
        qg = active(dom.get_state(0), *n)
        bg = [active(b, *n).copy() for b in dom.get_face_b(0)]
    q0 = hm.problem_state(p)
    o.set_state(q0)
    del q0
    rc, to, odts = o.run(10.0, 1, steps)
    assert s == steps and len(odts) == steps
    err = rel_l1(qg, active(o.get_q(0), *n))
    del qg
    bo = o.get_faceb(0)
    eb = [rel_l1(bg[c][None], active(bo[c], *n)[None])[0] for c in range(3)]
    dte = _dt_err(dts, odts)
    parity_record(case=f"blast3d_b_{n1}^3_fp64", steps=steps, max_rel_dt=dte, rel_l1_q=err, rel_l1_faceb=eb,
                  oracle_self_sensitivity=SENS_BLAST256 if n1 == 256 else None)
    if n1 == 256:
        bar = np.maximum(TOL_Q, 10.0 * SENS_BLAST256)
        assert dte <= 10.0 * SENS_BLAST256_DT, dte
        assert np.all(err <= bar), (err, bar)
        assert eb[0] <= TOL_Q and eb[1] <= TOL_Q and eb[2] <= bar[6], eb
        assert err[0] <= TOL_Q and err[4] <= TOL_Q and err[5] <= TOL_Q, err
    else:
        assert dte <= 1e-13, dte
        assert np.all(err <= TOL_Q), err
        assert max(eb) <= TOL_Q, eb
