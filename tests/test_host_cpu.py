"""Host-side logic of the product library that needs no GPU: the input.in
parser (src/parameters.cpp:7-160 semantics), the problem registry
(src/problem.cpp:7-37) and initial conditions (bit-equal to the reference's
restated ones), the new problems' properties, and the C ABI's exports."""
import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

from howtest import REPO, CPUOracle, active

hm = pytest.importorskip("how_mhd")


# ------------------------------------------------------------------ parser
def test_defaults_match_reference():
    p = hm.read_parameters("nx 4\nny 4\nnz 4\nnt 1\ntend 1.0\n")
    assert p.gam == 5.0 / 3.0 and p.cour == 0.4
    assert p.rhomin == 1e-12 and p.pgmin == 1e-12
    assert (p.xsize, p.ysize, p.zsize) == (1.0, 1.0, 1.0)
    assert list(p.bc) == [hm.HOW_BC_PERIODIC] * 3
    assert p.output_format == b"dat"
    assert p.dx == 0.25


def test_comments_aliases_and_unknown_keys(capfd):
    text = ("# a comment line\n"
            "gnx 8 # trailing comment\n"
            "ny 6\nnz 1\nnt 3\ntend 0.5\n"
            "frobnicate 12 13 14\n"          # unknown: warned, rest of line skipped
            "x1bc open\nproblem orszag_tang\npx 2\n")
    p = hm.read_parameters(text)
    assert (p.nx, p.ny, p.nz, p.nt, p.tend) == (8, 6, 1, 3, 0.5)
    assert p.bc[0] == hm.HOW_BC_OPEN
    assert p.problem == b"orszag_tang"
    assert "unknown parameter frobnicate" in capfd.readouterr().err


@pytest.mark.parametrize("text,msg", [
    ("nx 4\nny 4\nnz 0\nnt 1\ntend 1\n", "grid size"),
    ("nx 4\nny 4\nnz 4\nnt 0\ntend 1\n", "nt must be positive"),
    ("nx 4\nny 4\nnz 4\nnt 1\ntend 0\n", "tend must be positive"),
    ("nx 4\nny 4\nnz 4\nnt 1\ntend 1\nx2bc reflecting\n", "unknown x2bc"),
    ("nx 4\nny 4\nnz 4\nnt 1\ntend 1\nprecision half\n", "unknown precision"),
    ("nx 4\nny\n", "invalid value"),
])
def test_validation_errors_are_status_codes(text, msg):
    with pytest.raises(hm.HowError) as e:
        hm.read_parameters(text)
    assert msg in str(e.value)


def test_extension_keys():
    p = hm.read_parameters("nx 4\nny 4\nnz 4\nnt 1\ntend 1\nprecision mixed\nrouter on\nseed 99\npar3 2.5\n")
    assert p.precision == hm.HOW_PREC_MIXED and p.router == 1 and p.seed == 99
    assert p.problem_par[3] == 2.5


# ---------------------------------------------------------------- registry
def test_registry_lists_reference_and_new_problems():
    names = set(hm.list_problems())
    assert {"orszag_tang", "blast3d", "brio_wu", "mhd_rotor", "uniform", "mpi_smooth3d"} <= names
    assert {"alfven3d", "blast3d_b", "turb3d"} <= names


def test_unknown_problem_lists_available():
    p = hm.make_parameters(nx=4, ny=4, nz=4, nt=1, tend=1.0, problem="nope")
    with pytest.raises(hm.HowError) as e:
        hm.problem_state(p)
    assert "unknown problem = nope" in str(e.value) and "orszag_tang" in str(e.value)


def test_register_problem_from_python():
    def init(q, p):
        q[0, 3:-3, 3:-3, 3:-3] = 2.0
        q[7, 3:-3, 3:-3, 3:-3] = 3.0
    hm.register_problem("py_const", init)
    p = hm.make_parameters(nx=5, ny=4, nz=3, nt=1, tend=1.0, problem="py_const")
    q = hm.problem_state(p)
    assert np.all(active(q, 5, 4, 3)[0] == 2.0) and np.all(active(q, 5, 4, 3)[7] == 3.0)
    assert np.all(q[0, :3] == 0.0)   # ghosts untouched (zeroed)


@pytest.mark.parametrize("prob,n,gam", [
    ("orszag_tang", (24, 20, 1), 5.0 / 3.0), ("blast3d", (12, 10, 8), 5.0 / 3.0),
    ("brio_wu", (50, 1, 1), 2.0), ("mhd_rotor", (20, 24, 1), 1.4),
    ("uniform", (6, 5, 4), 5.0 / 3.0), ("mpi_smooth3d", (10, 8, 6), 5.0 / 3.0),
    ("blast3d_b", (14, 12, 10), 5.0 / 3.0)])
def test_initial_conditions_bit_equal_to_restatement(prob, n, gam):
    p = hm.make_parameters(nx=n[0], ny=n[1], nz=n[2], nt=1, tend=1.0, gam=gam, problem=prob)
    q = hm.problem_state(p)
    o = CPUOracle(*n, gam=gam)
    o.init_problem(prob)
    np.testing.assert_array_equal(active(q, *n), active(o.get_q(0), *n))


def test_alfven3d_is_exact_wave_state():
    n = 16
    p = hm.make_parameters(nx=n, ny=n, nz=n, nt=1, tend=1.0, problem="alfven3d")
    q = active(hm.problem_state(p), n, n, n)
    rho, B, v = q[0], q[4:7], q[1:4] / q[0]
    e1 = np.ones(3) / np.sqrt(3.0)
    Bpar = np.einsum("d,dijk->ijk", e1, B)
    Bperp = B - Bpar * e1[:, None, None, None]
    np.testing.assert_allclose(Bpar, 1.0, atol=1e-14)
    np.testing.assert_allclose(np.sqrt((Bperp ** 2).sum(0)), 0.1, atol=1e-14)
    np.testing.assert_allclose(v, -Bperp / np.sqrt(rho), atol=1e-14)   # travels along +e1
    np.testing.assert_allclose(rho, 1.0)


def test_turb3d_rms_and_solenoidal():
    n = 24
    p = hm.make_parameters(nx=n, ny=n, nz=n, nt=1, tend=1.0, problem="turb3d", seed=12345)
    q = active(hm.problem_state(p), n, n, n)
    v = q[1:4] / q[0]
    assert abs(np.sqrt((v ** 2).sum(0).mean()) - 0.5) < 1e-12
    k = np.fft.fftfreq(n) * n
    kx, ky, kz = np.meshgrid(k, k, k, indexing="ij")
    vh = [np.fft.fftn(v[d]) for d in range(3)]
    div = kx * vh[0] + ky * vh[1] + kz * vh[2]
    assert np.abs(div).max() < 1e-9 * np.abs(vh[0]).max()
    kk = np.sqrt(kx ** 2 + ky ** 2 + kz ** 2)
    power = sum(np.abs(x) ** 2 for x in vh)
    assert power[(kk < 1) | (kk > 4 + 1e-9)].sum() < 1e-20 * power.sum()
    q2 = active(hm.problem_state(p), n, n, n)
    np.testing.assert_array_equal(q, q2)   # seeded: reproducible


def test_blast3d_b_regions():
    n = 32
    p = hm.make_parameters(nx=n, ny=n, nz=n, nt=1, tend=1.0, problem="blast3d_b")
    q = active(hm.problem_state(p), n, n, n)
    np.testing.assert_allclose(q[4:6], 1.0 / np.sqrt(2.0))
    assert np.all(q[6] == 0.0)
    pg = (5.0 / 3.0 - 1.0) * (q[7] - 0.5 * (q[4:7] ** 2).sum(0))
    assert set(np.round(np.unique(pg), 12)) == {0.1, 10.0}


# --------------------------------------------------------------------- ABI
def test_library_exports_every_declared_function():
    header = (REPO / "include" / "how_mhd.h").read_text()
    declared = set(re.findall(r"^\s*(?:int|double|long|size_t|void\*|const char\*)\s+(how_\w+)\s*\(", header, re.M))
    assert len(declared) >= 30
    lib = ctypes.CDLL(hm.LIBRARY_PATH)
    missing = [f for f in sorted(declared) if not hasattr(lib, f)]
    assert not missing, missing


def test_context_creation_fails_cleanly_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    p = hm.make_parameters(nx=8, ny=8, nz=8, nt=1, tend=1.0, problem="uniform")
    with pytest.raises(hm.HowError) as e:
        hm.Domain(p)
    assert e.value.code == -5   # HOW_ERR_NODEVICE, not a crash or a CPU fallback
