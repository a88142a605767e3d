"""Measures the oracle's own sensitivity: the blast3d_b run (10 steps from
t = 0, floors 1e-6) from its initial state and from that state perturbed by
a seeded 1e-16 relative noise; prints the relative L1 per conserved variable
between the two and the max relative dt change.  The figures behind
SENS_BLAST256 in test_gpu_parity.py came from

    python tests/oracle_sensitivity.py 256      (about 11 GB, minutes on 8 cores)

Test infrastructure only (not collected by pytest)."""
import json
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
sys.path.insert(0, str(HERE.parent / "how-mhd-kokkos_b200"))
from howtest import CPUOracle, active, oracle_lib, rel_l1   # noqa: E402


def main(n):
    import how_mhd as hm
    oracle_lib().oracle_set_threads(os.cpu_count() or 1)
    p = hm.make_parameters(nx=n, ny=n, nz=n, nt=1, tend=10.0, problem="blast3d_b", rhomin=1e-6, pgmin=1e-6)
    q0 = hm.problem_state(p)
    res = []
    for pert in (0.0, 1e-16):
        q = q0.copy()
        if pert:
            a = active(q, n, n, n)
            a *= 1 + pert * np.random.default_rng(0).standard_normal(a.shape)
        o = CPUOracle(n, n, n, rhomin=1e-6, pgmin=1e-6)
        o.set_state(q)
        rc, t, dts = o.run(10.0, 1, 10)
        res.append((active(o.get_q(0), n, n, n).copy(), dts))
        del o
    print(json.dumps({"n": n, "rel_l1": rel_l1(res[1][0], res[0][0]).tolist(),
                      "dt": float(np.max(np.abs(res[1][1] - res[0][1]) / res[0][1]))}))


if __name__ == "__main__":
    main(int(sys.argv[1]) if len(sys.argv) > 1 else 256)
