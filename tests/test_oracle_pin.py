"""Pin the CPU restatement (oracle/how_oracle.cpp) to the reference itself.

1. Against the committed golden fixtures made by the reference's own sources
   (tests/golden/make_golden.py): bit-exact dt sequence, state and face B.
2. When the reference build oracle/_ref/how_ref is present (it travels with
   the repository snapshot; it is built from the reference checkout), against
   live runs: randomised states through single sweeps and whole steps,
   bit-exact.
"""
from pathlib import Path

import numpy as np
import pytest

from howtest import GOLDEN, REF_BIN, CPUOracle, active, oracle_lib, read_dump, run_ref, write_dump, write_input

FIXTURES = sorted(GOLDEN.glob("*.npz"))


@pytest.mark.parametrize("path", FIXTURES, ids=[p.stem for p in FIXTURES])
def test_oracle_matches_golden_bitwise(path):
    d = np.load(path)
    n = tuple(int(x) for x in d["n"])
    bc = tuple(str(x) for x in d["bc"])
    o = CPUOracle(*n, bc=bc, gam=float(d["gam"]))
    o.init_problem(str(d["problem"]))
    rc, t, dts = o.run(10.0, 1, int(d["steps"]))
    assert rc == 0
    np.testing.assert_array_equal(dts, d["dt"])
    np.testing.assert_array_equal(active(o.get_q(0), *n), d["q"])
    for b, name in zip(o.get_faceb(0), ("bxb", "byb", "bzb")):
        np.testing.assert_array_equal(active(b, *n), d[name])


needs_ref = pytest.mark.skipif(not REF_BIN.exists(), reason="reference build oracle/_ref/how_ref absent")


def _random_state(n, seed):
    """A smooth random state with positive density and pressure."""
    rng = np.random.default_rng(seed)
    P = tuple(x + 6 for x in n)
    q = np.zeros((8,) + P)
    a = active(q, *n)
    rho = 1.0 + 0.2 * rng.random(a.shape[1:])
    v = 0.3 * rng.standard_normal((3,) + a.shape[1:])
    B = 0.5 * rng.standard_normal((3,) + a.shape[1:])
    p = 1.0 + 0.3 * rng.random(a.shape[1:])
    gam = 5.0 / 3.0
    a[0] = rho
    a[1:4] = rho * v
    a[4:7] = B
    a[7] = p / (gam - 1.0) + 0.5 * rho * (v ** 2).sum(0) + 0.5 * (B ** 2).sum(0)
    return q


@needs_ref
@pytest.mark.parametrize("direction", ["x", "y", "z"])
def test_oracle_sweep_matches_reference_bitwise(tmp_path, direction):
    n = (12, 10, 8)
    bc = ("periodic", "open", "periodic")
    q = _random_state(n, 7)
    inp = write_input(tmp_path / "in.txt", nx=n[0], ny=n[1], nz=n[2], nt=1, tend=1.0,
                      problem="uniform", x1bc=bc[0], x2bc=bc[1], x3bc=bc[2])
    write_dump(tmp_path / "state.bin", {"q": q})
    dt = 1.0e-3
    ref = run_ref(inp, tmp_path / "out.bin", "--state", tmp_path / "state.bin", "--sweep", direction,
                  "--dt", repr(dt))
    o = CPUOracle(*n, bc=bc)
    o.set_state(q)
    d = "xyz".index(direction)
    q1, ca, cb = o.sweep(d, dt)
    np.testing.assert_array_equal(active(q1, *n), active(ref["q1"], *n))
    names = {0: ("fsy", "fsz"), 1: ("gsz", "gsx"), 2: ("hsx", "hsy")}[d]
    sl = [slice(3, n[0] + 3), slice(3, n[1] + 3), slice(3, n[2] + 3)]
    sl[d] = slice(2, n[d] + 3)
    for arr, nm in zip((ca, cb), names):
        np.testing.assert_array_equal(arr[tuple(sl)], ref[nm][tuple(sl)])


@needs_ref
def test_oracle_step_matches_reference_bitwise(tmp_path):
    n = (10, 9, 8)
    bc = ("open", "periodic", "periodic")
    q = _random_state(n, 11)
    inp = write_input(tmp_path / "in.txt", nx=n[0], ny=n[1], nz=n[2], nt=1, tend=10.0,
                      problem="uniform", x1bc=bc[0], x2bc=bc[1], x3bc=bc[2])
    write_dump(tmp_path / "state.bin", {"q": q})
    ref = run_ref(inp, tmp_path / "out.bin", "--state", tmp_path / "state.bin", "--steps", 3)
    o = CPUOracle(*n, bc=bc)
    o.set_state(q)
    rc, t, dts = o.run(10.0, 1, 3)
    np.testing.assert_array_equal(dts, ref["dt"])
    np.testing.assert_array_equal(active(o.get_q(0), *n), active(ref["q"], *n))
    for b, name in zip(o.get_faceb(0), ("bxb", "byb", "bzb")):
        np.testing.assert_array_equal(active(b, *n), active(ref[name], *n))


@needs_ref
def test_reference_dump_stages_equals_reference_ssprk(tmp_path):
    """The driver's call-for-call restatement of ssprk's stage loop (used for
    per-stage dumps) equals the reference's own ssprk."""
    n = (12, 12, 1)
    inp = write_input(tmp_path / "in.txt", nx=n[0], ny=n[1], nz=n[2], nt=1, tend=10.0, problem="orszag_tang")
    a = run_ref(inp, tmp_path / "a.bin", "--dump-stages")
    b = run_ref(inp, tmp_path / "b.bin", "--steps", 1)
    np.testing.assert_array_equal(active(a["final_q"], *n), active(b["q"], *n))


def test_oracle_ct_average_order_on_alfven():
    """On the 3-D circularly polarised Alfven wave the reference's two-point
    CT face average converges at second order, the four-point option at
    fourth (8^3 -> 16^3, one wave period)."""
    import how_mhd as hm
    lib = oracle_lib()

    def err(n, pts):
        T = float(1.0 / np.sqrt(3.0))
        p = hm.make_parameters(nx=n, ny=n, nz=n, nt=1, tend=T, gam=5.0 / 3.0, cour=0.4, problem="alfven3d")
        q0 = hm.problem_state(p)
        lib.oracle_set_ct_avg(pts)
        try:
            o = CPUOracle(n, n, n)
            o.set_state(q0)
            rc, t, _ = o.run(T)
            q = o.get_q(0)
        finally:
            lib.oracle_set_ct_avg(2)
        a0, a1 = active(q0, n, n, n), active(q, n, n, n)
        return np.mean([np.abs(a1[v] - a0[v]).mean() for v in (1, 2, 3, 4, 5, 6)])

    o2 = np.log2(err(8, 2) / err(16, 2))
    o4 = np.log2(err(8, 4) / err(16, 4))
    assert o2 < 2.2, o2
    assert o4 > 4.0, o4


@needs_ref
@pytest.mark.parametrize("prob,n", [("blast3d_b", (20, 18, 16)), ("alfven3d", (12, 10, 8)),
                                    ("turb3d", (16, 12, 10)), ("alfven3d", (24, 1, 1))])
def test_reference_build_problems_bit_equal_to_product(tmp_path, prob, n):
    """The benchmark problems the reference lacks are registered into the
    reference build through its own RegisterProblem (oracle/ref_problems.cpp);
    with default parameters their states equal the product's bit for bit, so
    the reference arm of the benchmark builds its state without the product."""
    hm = pytest.importorskip("how_mhd")
    inp = write_input(tmp_path / "in.txt", nx=n[0], ny=n[1], nz=n[2], nt=1, tend=1.0, problem=prob,
                      x1bc="periodic", x2bc="periodic", x3bc="periodic")
    d = run_ref(inp, tmp_path / "out.bin", "--steps", 0)
    p = hm.make_parameters(nx=n[0], ny=n[1], nz=n[2], nt=1, tend=1.0, problem=prob)
    np.testing.assert_array_equal(active(d["q"], *n), active(hm.problem_state(p), *n))
