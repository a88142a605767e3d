"""Learned WENO routing on decaying turbulence (problem turb3d: rho 1, p 1,
B = (0.5, 0, 0), seeded solenoidal velocity modes with 1 <= |k|/2pi <= 4 at
rms 0.5) at 64^3: mixed precision + learned routing against the plain FP64
method from the same state.  Bar: density relative L1 <= 1e-5; the CT keeps
max |div4 B| at round-off in both forms."""
import numpy as np
import pytest

from howtest import active
from test_gpu_mixed import div4

pytestmark = pytest.mark.gpu


def test_turbulence_routed_vs_plain(parity_record):
    import how_mhd as hm
    n = 64
    steps = 40
    out = {}
    for form, prec, router in (("fp64", "fp64", "off"), ("mixed+learned", "mixed", "on")):
        p = hm.make_parameters(nx=n, ny=n, nz=n, nt=1, tend=100.0, gam=5.0 / 3.0, cour=0.4, problem="turb3d",
                               precision=prec, router=router)
        with hm.Domain(p) as dom:
            dom.init_problem()
            if router == "on":
                dom.router_stats(reset=True)
            dom.run(0.0, steps)
            q = active(dom.get_state(0), n, n, n)
            b = dom.get_face_b(0)
            st = dom.router_stats() if router == "on" else None
        out[form] = (q, float(np.abs(div4(*b, (n, n, n), (p.dx, p.dy, p.dz))).max()), st)
    q64, dv64, _ = out["fp64"]
    qr, dvr, (full, cheap) = out["mixed+learned"]
    rho = float(np.abs(qr[0] - q64[0]).sum() / np.abs(q64[0]).sum())
    en = float(np.abs(qr[7] - q64[7]).sum() / np.abs(q64[7]).sum())
    frac = full / max(full + cheap, 1)
    parity_record(case="turb64_routed_vs_fp64", steps=steps, rho_l1=rho, energy_l1=en, full_weno_fraction=frac,
                  max_div_b_fp64=dv64, max_div_b_routed=dvr)
    assert rho <= 1e-5, rho
    assert 0.0 < frac <= 1.0, frac
    assert dv64 <= 1e-12 and dvr <= 1e-12, (dv64, dvr)
