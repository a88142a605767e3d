"""A small, self-contained case of the sweep kernel for profilers.

    python -m how_mhd.profile_case --n 128 --precision fp64 --router off --steps 2

advances the 3-D magnetised blast (blast3d_b) from the state at --t-start
(or a state saved by an earlier --save-state run) for --steps full steps (15
sweep launches each), then launches one x, one y and one z sweep on their own
(how_sweep).  Under a profiler, skip 15 * steps sweep launches to reach the
first of the three.  Prints the
per-phase cycle profile of each direction and the routing counters.
"""
import argparse
import json

import numpy as np

import how_mhd as hm


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--router", default="off", choices=["off", "on", "guard"])
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--t-start", type=float, default=0.0)
    ap.add_argument("--phases", action="store_true", help="also run the per-phase cycle profile")
    ap.add_argument("--save-state", default=None, help="write the state at --t-start (.npz) and stop")
    ap.add_argument("--load-state", default=None, help="start from a state written by --save-state")
    a = ap.parse_args(argv)
    n = a.n
    kw = dict(nx=n, ny=n, nz=n, nt=1, gam=5.0 / 3.0, cour=0.4, problem="blast3d_b", rhomin=1e-6, pgmin=1e-6)
    q = b = None
    if a.load_state:
        z = np.load(a.load_state)
        q, b, a.t_start = z["q"], [z["bx"], z["by"], z["bz"]], float(z["t"])
    elif a.t_start > 0:
        # the blast evolved to t_start by the mixed + learned-routing form
        with hm.Domain(hm.make_parameters(tend=a.t_start, precision="mixed", router="on", **kw)) as d:
            d.init_problem()
            d.run(0.0, -1)
            q, b = d.get_state(0), d.get_face_b(0)
        if a.save_state:
            np.savez(a.save_state, q=q, bx=b[0], by=b[1], bz=b[2], t=a.t_start)
            return
    p = hm.make_parameters(tend=1e3, precision=a.precision, router="on" if a.router == "on" else "off", **kw)
    with hm.Domain(p) as d:
        if q is None:
            d.init_problem()
        else:
            d.set_state(q)
            d.set_face_b(*b)
        if a.router == "guard":
            w, thr = hm.default_router()
            d.set_router(w, "guard", threshold=thr)
        t, _, _ = d.run(a.t_start, a.steps)
        dt = d.tstep()
        for k in range(3):
            d.sweep(k, dt)
        out = {"n": n, "precision": a.precision, "router": a.router, "t": t, "dt": dt}
        if a.router != "off":
            out["router_stats"] = d.router_stats(groups=True)
        if a.phases:
            out["phases"] = [d.sweep_phase_profile(k, dt).tolist() for k in range(3)]
        print(json.dumps(out))


if __name__ == "__main__":
    main()
