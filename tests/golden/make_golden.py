"""Generate the golden fixtures of tests/golden/ from the reference itself.

The reference's own sources, compiled unmodified against the project's Kokkos
shim (oracle/Makefile -> oracle/_ref/how_ref), run each case below; the
active-cell state, face B and dt sequence after the given number of steps are
stored as compressed .npz.  Run from the repository root:

    make -C oracle ref && python tests/golden/make_golden.py
"""
from __future__ import annotations

import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent))
from howtest import REF_BIN, run_ref, write_input  # noqa: E402

CASES = {
    # name: (problem, n, bc, gam, steps)
    "ot32_5": ("orszag_tang", (32, 32, 1), ("periodic",) * 3, 5.0 / 3.0, 5),
    "blast12_3": ("blast3d", (12, 12, 12), ("periodic",) * 3, 5.0 / 3.0, 3),
    "rotor24_open_5": ("mhd_rotor", (24, 24, 1), ("open", "open", "periodic"), 1.4, 5),
    "briowu64_10": ("brio_wu", (64, 1, 1), ("open",) * 3, 2.0, 10),
    "smooth_10x8x6_3": ("mpi_smooth3d", (10, 8, 6), ("periodic", "open", "periodic"), 5.0 / 3.0, 3),
}


def main():
    if not REF_BIN.exists():
        sys.exit(f"build the reference first: make -C oracle ref ({REF_BIN} missing)")
    with tempfile.TemporaryDirectory() as td:
        for name, (prob, n, bc, gam, steps) in CASES.items():
            inp = write_input(Path(td) / f"{name}.in", nx=n[0], ny=n[1], nz=n[2], nt=1, tend=10.0, gam=gam,
                              cour=0.4, problem=prob, x1bc=bc[0], x2bc=bc[1], x3bc=bc[2])
            d = run_ref(inp, Path(td) / f"{name}.bin", "--steps", steps)
            s = (slice(3, n[0] + 3), slice(3, n[1] + 3), slice(3, n[2] + 3))
            np.savez_compressed(HERE / f"{name}.npz", q=d["q"][(slice(None),) + s],
                                bxb=d["bxb"][s], byb=d["byb"][s], bzb=d["bzb"][s], dt=d["dt"],
                                problem=prob, n=np.array(n), bc=np.array(bc), gam=gam, steps=steps)
            print("wrote", name)


if __name__ == "__main__":
    main()
