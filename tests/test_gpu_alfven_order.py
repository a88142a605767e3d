"""Convergence on the smooth circularly polarised Alfven wave (3-D periodic
unit cube, wave vector 2 pi (1, 1, 1); after one wave period the exact
solution is the initial state).

The reference's CT flux terms average B_n v_t over the two cells of a face
(the 4-point weights with outer weights -0.0, src/ssprk.cpp:976-989), which
holds the transverse fields to second order on this wave; the oracle, which
follows the reference bit for bit, shows the same.  With ct_avg 4 (the
fourth-order face value) the FP64 path converges at order >= 4.  The 1-D
wave (no CT) is fifth order either way."""
import numpy as np
import pytest

from howtest import active

pytestmark = pytest.mark.gpu

PERIOD3 = float(1.0 / np.sqrt(3.0))   # wavelength 1/sqrt(3) at v_A = B_par / sqrt(rho) = 1


def _error(n, dims, precision="fp64", ct_avg=2):
    import how_mhd as hm
    nx, ny, nz = [n if d else 1 for d in dims]
    period = float(1.0 / np.sqrt(sum(dims)))
    p = hm.make_parameters(nx=nx, ny=ny, nz=nz, nt=1, tend=period, gam=5.0 / 3.0, cour=0.4,
                           problem="alfven3d", precision=precision, ct_avg=ct_avg)
    with hm.Domain(p) as d:
        d.init_problem()
        q0 = active(d.get_state(0), nx, ny, nz).copy()
        t, steps, _ = d.run(0.0, 10 ** 6)
        assert abs(t - period) < 1e-12
        q = active(d.get_state(0), nx, ny, nz)
    # L1 over the transverse momentum and field components
    return float(np.mean([np.abs(q[v] - q0[v]).mean() for v in (1, 2, 3, 4, 5, 6)]))


_ERRS = {}


def _errs(key):
    if key not in _ERRS:
        dims, prec, ct = key
        ns = (32, 64, 128) if sum(dims) == 3 else (64, 128, 256)
        _ERRS[key] = [_error(n, dims, prec, ct) for n in ns]
    return _ERRS[key]


def _orders(e):
    return [float(np.log2(e[i] / e[i + 1])) for i in range(len(e) - 1)]


def test_alfven3d_order_ct4_fp64():
    e = _errs(((1, 1, 1), "fp64", 4))
    assert _orders(e)[-1] >= 4.0, (e, _orders(e))


def test_alfven3d_reference_ct_is_second_order():
    e = _errs(((1, 1, 1), "fp64", 2))
    o = _orders(e)
    assert 1.8 <= o[-1] <= 2.2, (e, o)
    # and the 4-point average is far more accurate at every size
    e4 = _errs(((1, 1, 1), "fp64", 4))
    assert all(a < 0.1 * b for a, b in zip(e4[1:], e[1:])), (e4, e)


def test_alfven1d_order_fp64():
    e = _errs(((1, 0, 0), "fp64", 2))
    assert _orders(e)[-1] >= 4.0, (e, _orders(e))


def test_alfven3d_mixed_tracks_fp64():
    e64 = _errs(((1, 1, 1), "fp64", 4))
    em = _errs(((1, 1, 1), "mixed", 4))
    for a, b in zip(em, e64):
        assert abs(a - b) <= 0.05 * b + 1e-9, (em, e64)
