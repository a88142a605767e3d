"""Mixed precision (FP32 eigen-system / projection / WENO, FP64 accumulation,
CT and CFL) against the plain FP64 path, and the divergence the CT keeps at
round-off.  Bars: density and pressure relative L1 <= 1e-5 against FP64
after the run; max |div4 B| <= 1e-12 (4th-order face divergence, the
quantity the CT update preserves exactly, src/fluxct.cpp:848-876)."""
import numpy as np
import pytest

from howtest import active

pytestmark = pytest.mark.gpu


def div4(bx, by, bz, n, d):
    """sum_d [9/8 (b(i) - b(i-1)) - 1/24 (b(i+1) - b(i-2))] / h_d at active cells;
    bxb(i) is the face at i+1/2."""
    nx, ny, nz = n
    sx = slice(3, nx + 3)
    sy = slice(3, ny + 3)
    sz = slice(3, nz + 3)

    def D(b, axis, h):
        def sh(k):
            s = [sx, sy, sz]
            base = s[axis]
            s[axis] = slice(base.start + k, base.stop + k)
            return b[tuple(s)]
        return (9.0 / 8.0 * (sh(0) - sh(-1)) - 1.0 / 24.0 * (sh(1) - sh(-2))) / h
    out = 0.0
    if nx > 1:
        out = out + D(bx, 0, d[0])
    if ny > 1:
        out = out + D(by, 1, d[1])
    if nz > 1:
        out = out + D(bz, 2, d[2])
    return out


def _run(prob, n, precision, steps, **kw):
    import how_mhd as hm
    p = hm.make_parameters(nx=n[0], ny=n[1], nz=n[2], nt=1, tend=100.0, gam=5.0 / 3.0, cour=0.4,
                           problem=prob, precision=precision, **kw)
    with hm.Domain(p) as dom:
        dom.init_problem()
        t, s, dts = dom.run(0.0, steps, dts_cap=steps)
        return dom.get_state(0), dom.get_face_b(0), dts, p


def _pressure(q, gam=5.0 / 3.0):
    return (gam - 1.0) * (q[7] - 0.5 * (q[1] ** 2 + q[2] ** 2 + q[3] ** 2) / q[0]
                          - 0.5 * (q[4] ** 2 + q[5] ** 2 + q[6] ** 2))


@pytest.mark.parametrize("prob,n,steps,kw", [
    ("blast3d_b", (48, 48, 48), 40, dict(rhomin=1e-6, pgmin=1e-6)),
    ("orszag_tang", (128, 128, 1), 100, {}),
])
def test_mixed_vs_fp64(prob, n, steps, kw, parity_record):
    q64, b64, dts64, p = _run(prob, n, "fp64", steps, **kw)
    q32, b32, dts32, _ = _run(prob, n, "mixed", steps, **kw)
    a64, a32 = active(q64, *n), active(q32, *n)
    rho_err = np.abs(a32[0] - a64[0]).sum() / np.abs(a64[0]).sum()
    pg_err = np.abs(_pressure(a32) - _pressure(a64)).sum() / np.abs(_pressure(a64)).sum()
    assert rho_err <= 1e-5, rho_err
    assert pg_err <= 1e-5, pg_err
    np.testing.assert_allclose(dts32, dts64, rtol=1e-5)
    d = (p.dx, p.dy, p.dz)
    dvs = []
    for b in (b64, b32):
        scale = np.abs(np.array(b)).max() / min(x for x, m in zip(d, n) if m > 1)
        dvs.append((float(np.abs(div4(*b, n, d)).max()), float(scale)))
    parity_record(case=f"mixed_vs_fp64_{prob}", steps=steps, rho_l1=rho_err, p_l1=pg_err,
                  max_div_b_fp64=dvs[0][0], max_div_b_mixed=dvs[1][0], max_abs_b_over_dx=dvs[0][1])
    for dv, scale in dvs:
        assert dv <= 1e-12, (dv, scale)   # absolute, the north star's bar


def test_divb_roundoff_fp64_alfven():
    n = (32, 32, 32)
    q, b, dts, p = _run("alfven3d", n, "fp64", 10)
    dv = np.abs(div4(*b, n, (p.dx, p.dy, p.dz))).max()
    assert dv <= 1e-12, dv


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_divb_absolute_headline_size(precision, parity_record):
    """max |div4 B| <= 1e-12 absolute on the headline workload (blast3d_b
    256^3, |B| = 1, dx = 1/256) after 10 steps from t = 0, in both
    precisions (the CT update, in FP64 in both, keeps it at round-off)."""
    n = (256, 256, 256)
    q, b, dts, p = _run("blast3d_b", n, precision, 10, rhomin=1e-6, pgmin=1e-6)
    del q
    dv = float(np.abs(div4(*b, n, (p.dx, p.dy, p.dz))).max())
    parity_record(case=f"divb_blast256_{precision}", steps=10, max_div_b=dv,
                  max_div_b_over_b_per_dx=dv / (float(np.abs(np.array(b)).max()) / p.dx))
    assert dv <= 1e-12, dv
