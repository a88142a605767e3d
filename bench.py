#!/usr/bin/env python
"""bench.py -- zone-cycles/s of the HOW-MHD time step on B200.

Workload (the headline configuration): 3-D MHD blast, 256^3 periodic cube,
rho = 1, p = 10 inside r < 0.1 and 0.1 outside, B = (1, 1, 0)/sqrt 2, gam 5/3,
cour 0.4, floors 1e-6 (problem `blast3d_b`).  One bench step = one CFL
reduction (tstep) + one SSPRK(5,4) step (5 stages x 3 fused WENO sweeps + CT +
prot + ghost fills) over the whole domain; 1 zone-cycle = one active zone
advanced by one step.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--n 256] [--t-start 0.05] [--no-fast] [--no-e2e] [--no-cpu-baseline]

The timed steps start from the blast evolved to t_start.  `value` is the plain
FP64 method (the reference's), device-timed with the state resident in HBM;
`mixed_learned` is the mixed-precision + learned-routing form over the same
steps from the same state, with its density / energy L1 against the FP64
leg, max |div B| and the fraction of interfaces sent to full WENO.  `e2e`
goes through the C ABI with host (pinned) buffers: upload q + face B, tstep,
ssprk, download, every step.  Under torchrun each rank advances its own
replica (the path has no data exchange at one domain per GPU), time = max
over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO / "how-mhd-kokkos_b200"))

METRIC = "zone-cycles/s, 256^3 blast: plain FP64 vs mixed+learned, same L1 err, 1 B200"
UNIT = "zone-cycles/s"
# Algorithmic FP64 operations (add/sub/mul/div/sqrt/max/abs = 1 each), counted
# by instantiating the CPU restatement's cell/interface kernels on a counting
# scalar: 3,088 per zone per directional sweep (primitives 21, centre 71,
# interface eigenvectors 527, 7 x WENO field 332, 7 x back-projection 14,
# 7 x update 3, CT terms 26); per zone-cycle 5 x (3 x 3,088 + RK 46 + CT 147
# + prot 25) + stage-5 base 48 + tstep 60 = 47,518.
SWEEP_FLOP_PER_ZONE = 3088
FLOP_PER_ZONE_CYCLE = 47518
REF_SAMPLE_N = 64


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=None, help="cells per axis (default 256; 384 for --workload turbulence)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--t-start", type=float, default=0.05,
                    help="simulated time the timed steps start from (the blast evolved there first)")
    ap.add_argument("--no-fast", action="store_true", help="skip the mixed-precision + learned-routing leg")
    ap.add_argument("--workload", default="blast", choices=["blast", "ensemble", "accuracy", "output", "turbulence"],
                    help="ensemble: 64 uneven 2-D/1-D runs batched vs advanced one by one; "
                         "accuracy: whole blast run to --tend in every precision / routing form; "
                         "output: dump files (how_output) of the blast state, .vts and .dat; "
                         "turbulence: learned routing on decaying turbulence (turb3d, --n 384)")
    ap.add_argument("--out-dir", default="/tmp/how_dumps", help="--workload output: where the dumps go")
    ap.add_argument("--tend", type=float, default=0.2, help="end time of --workload accuracy")
    ap.add_argument("--forms", default="",
                    help="--workload accuracy: ';'-separated subset of the forms after fp64 (default: all)")
    ap.add_argument("--ref-sizes", default="128",
                    help="--impl reference: comma-separated larger sample sizes whose per-zone rate is "
                         "reported beside the 64^3 one (256 needs ~30 GB of host memory and minutes)")
    ap.add_argument("--t-start2", type=float, default=0.15,
                    help="second snapshot of the mixed + learned leg (0: none), where the shock front is larger")
    ap.add_argument("--turb-steps", type=int, default=100,
                    help="--workload turbulence: steps of each form from t = 0 (timed after --warmup)")
    return ap.parse_args()


def dist_info():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def workload_text(n, precision, tend=1.0e3, router="off"):
    # tend far beyond the timed steps so no step is shortened by the output clamp
    return (f"nx {n}\nny {n}\nnz {n}\nnt 1\ntend {tend!r}\ngam 1.6666666666666667\ncour 0.4\n"
            f"problem blast3d_b\nx1bc periodic\nx2bc periodic\nx3bc periodic\n"
            f"rhomin 1e-6\npgmin 1e-6\nprecision {precision}\nrouter {router}\n")


# ------------------------------------------------------------------ clocks
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, dev_id):
        self.dev_id = dev_id
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.dev_id}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        sm, smax, reasons = [], [], set()
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[3:7]):
                if v.lower() in ("active", "1"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "samples": len(sm),
                "reasons": sorted(reasons)}


def device_id_for_smi(local):
    import torch
    try:
        u = str(torch.cuda.get_device_properties(local).uuid)
        return u if u.startswith("GPU-") else "GPU-" + u
    except Exception:   # noqa: BLE001
        vis = os.environ.get("CUDA_VISIBLE_DEVICES")
        return vis.split(",")[local] if vis else str(local)


# -------------------------------------------------------------- CPU baseline
def ref_binary():
    b = REPO / "oracle" / "_ref" / "how_ref"
    return b if b.exists() else None


def reference_input(n):
    """input.in of the workload at n^3 with the reference's own keys only
    (src/parameters.cpp:46-111), so its parser has nothing to warn about."""
    return (f"nx {n}\nny {n}\nnz {n}\nnt 1\ntend 1000.0\ngam 1.6666666666666667\ncour 0.4\n"
            f"problem blast3d_b\nx1bc periodic\nx2bc periodic\nx3bc periodic\nrhomin 1e-6\npgmin 1e-6\n")


def run_reference_sample(n, steps, warmup, threads, timeout=3600):
    """Time the reference's own CPU path on blast3d_b n^3: oracle/_ref/how_ref,
    the reference's src/*.cpp built from its sources, which makes the initial
    state itself (the benchmark problems are registered into its registry
    through its RegisterProblem, oracle/ref_problems.cpp) and runs `warmup`
    untimed then `steps` timed main-loop steps.  Returns a dict (zone-cycles/s,
    kind "reference", peak RSS of that process).  If the reference build is
    absent or fails, its return code and stderr are logged and the oracle port
    (oracle/_build/liboracle.so) is timed instead (kind "port")."""
    binp = ref_binary()
    why = "reference build oracle/_ref/how_ref absent"
    if binp is not None:
        with tempfile.TemporaryDirectory() as td:
            inp = Path(td) / "in.txt"
            inp.write_text(reference_input(n))
            out, err = Path(td) / "out.txt", Path(td) / "err.txt"
            env = dict(os.environ, OMP_NUM_THREADS=str(threads))
            with open(out, "w") as fo, open(err, "w") as fe:
                proc = subprocess.Popen([str(binp), str(inp), "/dev/null", "--steps", str(steps), "--warmup",
                                         str(warmup), "--time-only", "--threads", str(threads)],
                                        stdout=fo, stderr=fe, env=env)
                t0 = time.perf_counter()
                while True:
                    pid, status, ru = os.wait4(proc.pid, os.WNOHANG)
                    if pid:
                        break
                    if time.perf_counter() - t0 > timeout:
                        proc.kill()
                        pid, status, ru = os.wait4(proc.pid, 0)
                        break
                    time.sleep(0.05)
            rc = os.waitstatus_to_exitcode(status)
            if rc == 0:
                js = json.loads(out.read_text().strip().splitlines()[-1])
                return {"zone_cycles_per_s": js["zone_cycles_per_s"], "kind": "reference", "n": n,
                        "steps": steps, "warmup": warmup, "threads": threads, "wall_s": js["wall_s"],
                        "peak_rss_gb": ru.ru_maxrss / 1e6}
            why = f"reference build exited {rc}: {err.read_text()[-400:]!r}"
    print(f"bench: {why}; timing the oracle port instead", file=sys.stderr, flush=True)
    sys.path.insert(0, str(REPO / "tests"))
    from howtest import CPUOracle, oracle_lib
    oracle_lib().oracle_set_threads(threads)
    o = CPUOracle(n, n, n, gam=5.0 / 3.0, rhomin=1e-6, pgmin=1e-6)
    o.init_problem("blast3d_b")
    for _ in range(warmup):
        o.ssprk(o.tstep())
    t0 = time.perf_counter()
    for _ in range(steps):
        o.ssprk(o.tstep())
    el = time.perf_counter() - t0
    return {"zone_cycles_per_s": n ** 3 * steps / el, "kind": "port", "n": n, "steps": steps, "warmup": warmup,
            "threads": threads, "wall_s": el, "why_port": why}


def sample_text(r):
    who = "the reference's own sources (oracle/_ref/how_ref)" if r["kind"] == "reference" else "the oracle port"
    return (f"blast3d_b {r['n']}^3 from t = 0 (the headline problem at a size the host finishes in seconds; the "
            f"reference's per-zone work does not depend on the state), {r['steps']} timed SSPRK step(s) after "
            f"{r['warmup']} warm-up, {r['threads']} OpenMP threads, {who}")


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def headline_config(n, world):
    """`config` of the headline workload, shared by both arms."""
    return {"workload": f"3-D MHD blast {n}^3 (blast3d_b), periodic, gam 5/3, cour 0.4, floors 1e-6; "
                        f"SSPRK(5,4) + characteristic WENO5/LLF + 4th-order CT; `value` = plain FP64, "
                        f"`mixed_learned` = FP32 characteristic part + learned WENO routing",
            "n": n, "parallelism": "replicas" if world > 1 else "single",
            "l2": "state 12.5 GB per replica >> 126 MB L2: every step streams from HBM, no flush"}


# ---------------------------------------------------------------- reference arm
def bench_reference(args):
    """The reference's own CPU implementation of the time step, timed on the
    host cores: each bench step is one SSPRK step of a bounded sample of the
    headline workload (blast3d_b at REF_SAMPLE_N^3); the per-zone rate at
    larger samples (--ref-sizes) is reported beside it."""
    world, rank, local = dist_info()
    if rank != 0:
        return 0
    threads = host_threads()
    t0 = time.perf_counter()
    main = run_reference_sample(REF_SAMPLE_N, max(args.steps, 1), args.warmup, threads)
    zcs = main["zone_cycles_per_s"]
    sizes = {}
    for m in [int(x) for x in args.ref_sizes.split(",") if x.strip()]:
        if m == REF_SAMPLE_N:
            continue
        sizes[f"{m}^3"] = run_reference_sample(m, 2 if m <= 128 else 1, 1 if m <= 128 else 0, threads)
    n3 = REF_SAMPLE_N ** 3
    line = {
        "impl": "reference", "metric": METRIC, "value": zcs, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * n3 / zcs,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": headline_config(args.n, world),
        "cpu_baseline": {"value": zcs, "unit": UNIT, "cores": threads, "kind": main["kind"],
                         "sample": sample_text(main)},
        "e2e": {"value": zcs, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "sample": main,
        "larger_samples": sizes,
        "wall_s": time.perf_counter() - t0,
    }
    print(json.dumps(line), flush=True)
    return 0


# --------------------------------------------------------- replica helpers
def max_over_ranks(x, world, device):
    """Max of a per-rank scalar over all ranks (the timing rule: the slowest
    replica sets the time).  `device` is "cuda" under NCCL, "cpu" under gloo."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(world, zones, steps, max_ms):
    """Whole-job zone-cycles/s: every replica advances `zones` for `steps`."""
    return world * zones * steps / (max_ms * 1e-3)


# ------------------------------------------------------------------ our arm
def load_traffic_profile(precision):
    f = REPO / "profiles" / "sweep_traffic.json"
    if not f.exists():
        return None
    try:
        d = json.loads(f.read_text())
        return d.get(precision, d.get("fp64"))
    except Exception:   # noqa: BLE001
        return None


def div4_max(b, n, d):
    """max |div B| of face B with the 4th-order face difference the CT update
    preserves (src/fluxct.cpp:848-876), over active cells."""
    import numpy as np
    s = slice(3, n + 3)

    def D(f, axis):
        def sh(k):
            sl = [s, s, s]
            sl[axis] = slice(3 + k, n + 3 + k)
            return f[tuple(sl)]
        return (9.0 / 8.0 * (sh(0) - sh(-1)) - 1.0 / 24.0 * (sh(1) - sh(-2))) / d
    return float(np.abs(D(b[0], 0) + D(b[1], 1) + D(b[2], 2)).max())


def div_report(b, n, dx):
    """max |div4 B| and that value relative to max |B| / dx (the size of one
    face-B difference quotient, i.e. the round-off scale of the measure)."""
    import numpy as np
    dv = div4_max(b, n, dx)
    bmax = float(max(np.abs(x).max() for x in b))
    return {"max_div_b": dv, "max_div_b_rel": dv / (bmax / dx) if bmax > 0 else None}


def bench_ours(args):
    import ctypes
    import numpy as np
    import torch
    import how_mhd as hm

    world, rank, local = dist_info()
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    n = args.n
    fp64_peak = ctypes_peak(hm)
    s_act = slice(3, n + 3)

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
        torch.cuda.synchronize()

    # The timed steps start from the blast at t_start (and, for the second
    # snapshot, t_start2), evolved by the fast path so every leg starts from
    # the same mid-run state with a shock in the box.
    t0_prep = time.perf_counter()
    snaps = []   # (t, q, face B)
    targets = [t for t in (args.t_start, args.t_start2 if not args.no_fast else 0.0) if t > 0]
    if targets:
        # each snapshot: a run with tend = that time (the main loop's clamp
        # lands on it exactly), continued from the previous snapshot
        t_now, q_now, b_now = 0.0, None, None
        for tt in sorted(targets):
            pp = hm.read_parameters(workload_text(n, "mixed", tend=tt, router="on"))
            with hm.Domain(pp) as d:
                if q_now is None:
                    d.init_problem()
                else:
                    d.set_state(q_now)
                    d.set_face_b(*b_now)
                t_now, _, _ = d.run(t_now, -1)
                q_now, b_now = d.get_state(0), d.get_face_b(0)
            snaps.append((t_now, q_now, b_now))
    else:
        snaps.append((0.0, None, None))
    prep_s = time.perf_counter() - t0_prep

    def make_domain(precision, router, snap):
        p = hm.read_parameters(workload_text(n, precision, router=router))
        dom = hm.Domain(p)
        if snap[1] is not None:
            dom.set_state(snap[1])
            dom.set_face_b(*snap[2])
        else:
            dom.init_problem()
        return p, dom

    def timed_leg(dom, t_start, clocks_too):
        """warm-up, then exactly K steps between barriers, CUDA events on the
        library's stream; returns ms, launches, sweep ms, sweep launches, clocks."""
        stream = torch.cuda.ExternalStream(dom.stream)
        t_sim, _, _ = dom.run(t_start, args.warmup)
        barrier()
        sampler = ClockSampler(device_id_for_smi(local)) if (rank == 0 and clocks_too) else None
        if sampler:
            sampler.start()
            time.sleep(0.5)
        hm.lib().how_set_kernel_timing(dom._h, 1)
        l0 = dom.kernel_launches
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        barrier()
        # an NVTX range around the timed steps, so a profiler can select
        # their launches alone (ncu --nvtx --nvtx-include "timed_steps/")
        torch.cuda.nvtx.range_push("timed_steps")
        e0.record(stream)
        dom.run(t_sim, args.steps)
        e1.record(stream)
        torch.cuda.nvtx.range_pop()
        barrier()
        ms = e0.elapsed_time(e1)
        launches = dom.kernel_launches - l0
        sweep_ms = ctypes.c_double()
        sweep_n = ctypes.c_long()
        hm.lib().how_get_kernel_timing(dom._h, ctypes.byref(sweep_ms), ctypes.byref(sweep_n))
        hm.lib().how_set_kernel_timing(dom._h, 0)
        clocks = sampler.stop() if sampler else None
        return max_over_ranks(ms, world, "cuda"), launches, sweep_ms.value, sweep_n.value, clocks

    def fp64_leg(snap, clocks_too, with_e2e):
        p, dom = make_domain("fp64", "off", snap)
        ms, launches, sweep_ms, sweep_n, clocks = timed_leg(dom, snap[0], clocks_too)
        value = replica_value(world, n ** 3, args.steps, ms)
        ref = None
        if rank == 0:
            q64 = dom.get_state(0)
            b64 = dom.get_face_b(0)
            ref = (q64[0, s_act, s_act, s_act].copy(), q64[7, s_act, s_act, s_act].copy(), div_report(b64, n, p.dx))
            del q64, b64
        e2e = None
        if with_e2e:
            stream = torch.cuda.ExternalStream(dom.stream)
            shp = (8,) + tuple(p.shape)
            qh = torch.empty(shp, dtype=torch.float64, pin_memory=True).numpy()
            bh = [torch.empty(tuple(p.shape), dtype=torch.float64, pin_memory=True).numpy() for _ in range(3)]
            dom.get_state(0, out=qh)
            dom.get_face_b_into(*bh)
            barrier()
            f0 = torch.cuda.Event(enable_timing=True)
            f1 = torch.cuda.Event(enable_timing=True)
            f0.record(stream)
            for _ in range(args.steps):
                dom.set_state(qh)
                dom.set_face_b(*bh)
                dt = dom.tstep()
                dom.ssprk(dt)
                dom.get_state(0, out=qh)
                dom.get_face_b_into(*bh)
            f1.record(stream)
            barrier()
            ems = max_over_ranks(f0.elapsed_time(f1), world, "cuda")
            nbytes = 8 * int(np.prod(shp)) + 3 * 8 * int(np.prod(p.shape))
            e2e = {"value": world * n ** 3 * args.steps / (ems * 1e-3), "unit": UNIT,
                   "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes,
                   "ms_per_step": ems / args.steps, "path": "plain FP64 through the C ABI (how_set_state, "
                                                             "how_tstep, how_ssprk, how_get_state)"}
            del qh, bh
        dom.close()
        return value, ms, launches, sweep_ms, sweep_n, clocks, ref, e2e

    def fast_leg(snap, ref, value64, refresh=5):
        pf, domf = make_domain("mixed", "on", snap)
        if refresh != 5:
            domf.set_router_refresh(refresh)
        domf.router_stats(reset=True)
        fms, flaunch, fsw_ms, fsw_n, _ = timed_leg(domf, snap[0], False)
        full, cheap = domf.router_stats()
        fvalue = replica_value(world, n ** 3, args.steps, fms)
        out = None
        if rank == 0:
            qf = domf.get_state(0)
            bf = domf.get_face_b(0)
            rf = qf[0, s_act, s_act, s_act]
            ef = qf[7, s_act, s_act, s_act]
            out = {
                "t_start": snap[0], "value": fvalue, "unit": UNIT, "ms_per_step": fms / args.steps,
                "speedup_vs_plain_fp64": fvalue / value64,
                "full_weno_fraction": full / max(full + cheap, 1),
                "l1_rho_vs_fp64": float(np.abs(rf - ref[0]).sum() / np.abs(ref[0]).sum()),
                "l1_energy_vs_fp64": float(np.abs(ef - ref[1]).sum() / np.abs(ref[1]).sum()),
                "gpu_launches": flaunch, "sweep_avg_ms": fsw_ms / max(fsw_n, 1),
            }
            out.update(div_report(bf, n, pf.dx))
            del qf, bf
        domf.close()
        return out

    # ---- snapshot 1: plain FP64 (the reference's method), e2e, the fast form
    value, ms, launches, sweep_ms, sweep_n, clocks, ref1, e2e = fp64_leg(snaps[0], True, not args.no_e2e)
    fast = None
    if not args.no_fast:
        fast = fast_leg(snaps[0], ref1, value)
        every = fast_leg(snaps[0], ref1, value, refresh=1)
        if rank == 0:
            w, thr = hm.default_router()
            fast["router_threshold"] = thr
            fast["note"] = ("same start state and step count as the plain FP64 leg; L1 over active cells; the "
                            "network decides once per step, the guard every stage")
            fast["decisions_every_stage"] = {k: every[k] for k in ("value", "ms_per_step", "speedup_vs_plain_fp64",
                                                                   "full_weno_fraction", "l1_rho_vs_fp64")}
        # ---- snapshot 2: the same comparison where the shock front is larger
        if len(snaps) > 1:
            v2, ms2, _, sw2, swn2, _, ref2, _ = fp64_leg(snaps[1], False, False)
            f2 = fast_leg(snaps[1], ref2, v2)
            if rank == 0:
                f2["plain_fp64"] = {"value": v2, "ms_per_step": ms2 / args.steps,
                                    "sweep_avg_ms": sw2 / max(swn2, 1), **ref2[2]}
                fast["second_snapshot"] = f2

    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0

    avg_sweep_ms = sweep_ms / max(sweep_n, 1)
    achieved = SWEEP_FLOP_PER_ZONE * n ** 3 / (avg_sweep_ms * 1e-3) / 1e12
    traffic = None
    tp = load_traffic_profile("fp64")
    if tp and "dram_bytes_per_zone" in tp:
        traffic = tp["dram_bytes_per_zone"] * n ** 3
    roofline = {
        "bound": "fp64", "unit": "TFLOP/s", "kernel": "k_sweep (fused directional WENO sweep), plain FP64",
        "achieved": achieved, "peak": fp64_peak, "frac": achieved / fp64_peak if fp64_peak else None,
        "peak_source": "measured live: FP64 FMA-pipe probe (how_measure_fp64_peak), of measured",
        "flop_per_launch": SWEEP_FLOP_PER_ZONE * n ** 3, "avg_launch_ms": avg_sweep_ms,
        "launches_timed": sweep_n, "share_of_step": sweep_ms / ms if ms else None,
        "traffic": traffic,
        "step_frac": value / world * FLOP_PER_ZONE_CYCLE / (fp64_peak * 1e12) if fp64_peak else None,
    }
    cpu = None
    if not args.no_cpu_baseline and world == 1:
        r = run_reference_sample(REF_SAMPLE_N, 3, 1, host_threads())
        cpu = {"value": r["zone_cycles_per_s"], "unit": UNIT, "cores": r["threads"], "kind": r["kind"],
               "sample": sample_text(r)}
    config = headline_config(n, world)
    config["t_start"] = snaps[0][0]
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": config,
        "prep_s": prep_s,
        "plain_fp64_div_b": ref1[2],
        "roofline": roofline,
        "mixed_learned": fast,
        "cpu_baseline": cpu,
        "e2e": e2e,
        "gpu_launches": launches,
        "clocks": clocks,
    }
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------- ensemble arm
def ensemble_members(hm, seed=2024):
    """The batched-ensemble workload: 24 Orszag-Tang vortices and 24 MHD rotors
    at sizes drawn from {64^2, 128^2, 256^2, 512^2} (gamma ~ U[1.4, 1.7] for
    the vortices), 16 Brio-Wu tubes of nx in {400, 800, 1600} (gamma 2, open)."""
    import numpy as np
    rng = np.random.default_rng(seed)
    sizes = [64, 128, 256, 512]
    P = hm.make_parameters
    out = []
    for _ in range(24):
        n = int(rng.choice(sizes))
        out.append(P(nx=n, ny=n, nz=1, nt=1, tend=0.5, gam=float(rng.uniform(1.4, 1.7)), cour=0.4,
                     problem="orszag_tang"))
    for _ in range(24):
        n = int(rng.choice(sizes))
        out.append(P(nx=n, ny=n, nz=1, nt=1, tend=0.15, gam=1.4, cour=0.4, problem="mhd_rotor",
                     x1bc="open", x2bc="open", x3bc="periodic"))
    for _ in range(16):
        n = int(rng.choice([400, 800, 1600]))
        out.append(P(nx=n, ny=1, nz=1, nt=1, tend=0.1, gam=2.0, cour=0.4, problem="brio_wu",
                     x1bc="open", x2bc="open", x3bc="open"))
    return out


def bench_ensemble(args):
    """Aggregate zone-cycles/s of the 64-member ensemble over K steps of every
    member: batched (one launch per kernel for all members, one CUDA graph per
    step, autotuned tile shapes) against the same members advanced one by one
    through how_run.  Replicas only under torchrun."""
    import torch
    import how_mhd as hm
    world, rank, local = dist_info()
    torch.cuda.set_device(local)
    members = ensemble_members(hm)
    zones = sum(p.nx * p.ny * p.nz for p in members)
    def events(stream):
        s = torch.cuda.ExternalStream(stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        return s, e0, e1

    with hm.Ensemble(members) as e:
        e.init()
        e.run(args.warmup + 3)               # autotune (3 steps) + warm-up
        torch.cuda.synchronize()
        s, e0, e1 = events(e.stream)
        t0 = time.perf_counter()
        e0.record(s)
        e.run(args.steps)
        e1.record(s)
        torch.cuda.synchronize()
        ens_host_s = time.perf_counter() - t0
        ens_s = e0.elapsed_time(e1) * 1e-3
        shapes, sweep_ms = e.shapes()
        launches = e.graph_launches
    # one by one, same K steps per member (each with its own warm-up), each
    # member's steps timed with events on its own stream, summed
    seq_s = 0.0
    for p in members:
        with hm.Domain(p) as d:
            d.init_problem()
            t, _, _ = d.run(0.0, args.warmup)
            d.sync()
            s, e0, e1 = events(d.stream)
            e0.record(s)
            d.run(t, args.steps)
            e1.record(s)
            d.sync()
            seq_s += e0.elapsed_time(e1) * 1e-3
    if rank != 0:
        return 0
    value = world * zones * args.steps / ens_s
    line = {
        "metric": "zone-cycles/s, batched ensemble of 64 uneven 2-D/1-D runs, 1 B200", "value": value,
        "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * ens_s / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "24 Orszag-Tang + 24 MHD rotors at {64..512}^2, 16 Brio-Wu at nx {400,800,1600}",
                   "members": len(members), "zones": zones,
                   "timing": "CUDA events on the ensemble's stream (batched) and on each member's stream (one by one, "
                             "summed); both include the host-side loop around the launches",
                   "host_clock_s": ens_host_s},
        "one_by_one": {"value": world * zones * args.steps / seq_s, "unit": UNIT, "seconds": seq_s},
        "speedup_vs_one_by_one": seq_s / ens_s,
        "tile_shapes": {name: hm.Ensemble.shape_info(d, s) for d, (name, s) in enumerate(zip("xyz", shapes))},
        "autotune_sweep_ms": sweep_ms.tolist(),
        "graph_launches": launches,
    }
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------- accuracy arm
def bench_accuracy(args):
    """The blast from t = 0 to --tend in plain FP64, mixed precision, mixed +
    learned routing and mixed + guard-only routing: density / energy L1 of each
    against FP64, max |div B|, ms per step and the fraction of interfaces sent
    to full WENO."""
    import numpy as np
    import torch
    import how_mhd as hm
    world, rank, local = dist_info()
    torch.cuda.set_device(local)
    n = args.n
    s = slice(3, n + 3)
    w, thr = hm.default_router()
    forms = [("fp64", "fp64", None, 5), ("mixed", "mixed", None, 5), ("mixed+learned", "mixed", "learned", 5),
             ("mixed+learned, decisions every stage", "mixed", "learned", 1),
             ("mixed+learned, decisions every two steps", "mixed", "learned", 10),
             ("mixed+guard", "mixed", "guard", 5)]
    if args.forms:
        keep = {f.strip() for f in args.forms.split(";")}
        forms = [f for f in forms if f[0] == "fp64" or f[0] in keep]   # FP64 is the reference
    out, ref = {}, None
    for name, prec, mode, refresh in forms:
        p = hm.read_parameters(workload_text(n, prec, tend=args.tend))
        with hm.Domain(p) as d:
            d.init_problem()
            if mode:
                d.set_router(w, mode, threshold=thr)
                d.set_router_refresh(refresh)
            d.sync()
            t0 = time.perf_counter()
            t, steps, _ = d.run(0.0, -1)
            d.sync()
            el = time.perf_counter() - t0
            q = d.get_state(0)
            b = d.get_face_b(0)
            st = d.router_stats() if mode else None
        rho, en = q[0, s, s, s].copy(), q[7, s, s, s].copy()
        del q
        r = {"steps": steps, "t": t, "ms_per_step": 1e3 * el / steps, "zone_cycles_per_s": n ** 3 * steps / el,
             "max_div_b": div4_max(b, n, p.dx), "max_abs_b": float(max(np.abs(x).max() for x in b))}
        if st:
            r["full_weno_fraction"] = st[0] / max(st[0] + st[1], 1)
        if ref is None:
            ref = (rho, en)
        else:
            r["l1_rho_vs_fp64"] = float(np.abs(rho - ref[0]).sum() / np.abs(ref[0]).sum())
            r["l1_energy_vs_fp64"] = float(np.abs(en - ref[1]).sum() / np.abs(ref[1]).sum())
        out[name] = r
        del b
    if rank == 0:
        print(json.dumps({"workload": f"blast3d_b {n}^3, t = 0 .. {args.tend}", "router_threshold": thr,
                          "timing": "host clock around the synchronised run (tstep + ssprk every step)",
                          "forms": out}), flush=True)
    return 0


# --------------------------------------------------------------- output arm
def bench_output(args):
    """Dump files of the blast state at --n: how_output in both formats,
    host clock around each synchronous call (device slab kernels, copies and
    file writes), the best of three, with the file size and write rate.  The
    reference writes the same files from host memory (src/output.cpp)."""
    import os
    import torch
    import how_mhd as hm
    world, rank, local = dist_info()
    torch.cuda.set_device(local)
    if rank != 0:
        return 0
    n = args.n
    out = {}
    for fmt in ("vts", "dat"):
        p = hm.read_parameters(workload_text(n, "fp64") + f"output_format {fmt}\n")
        with hm.Domain(p) as d:
            d.init_problem()
            d.run(0.0, 2)
            d.sync()
            best = None
            for _ in range(3):
                t0 = time.perf_counter()
                path = d.output(2, 0.0, args.out_dir)
                el = time.perf_counter() - t0
                best = el if best is None else min(best, el)
            size = os.path.getsize(path)
            os.remove(path)
        out[fmt] = {"s_per_dump": best, "bytes": size, "gb_per_s": size / best / 1e9}
    print(json.dumps({"workload": f"dump files of blast3d_b {n}^3 (how_output)", "timing": "host clock, best of 3",
                      "out_dir": args.out_dir, "formats": out}), flush=True)
    return 0


# ------------------------------------------------------------ turbulence arm
def bench_turbulence(args):
    """Learned WENO routing on decaying turbulence (problem turb3d: rho 1, p 1,
    B = (0.5, 0, 0), velocity a seeded sum of solenoidal Fourier modes with
    1 <= |k|/2pi <= 4 at rms 0.5) on a periodic --n^3 cube (384 by default).
    The plain FP64 method and mixed precision + learned routing each take
    --warmup untimed and --turb-steps device-timed steps from the same seeded
    state; reported: zone-cycles/s of both, the fraction of interfaces routed
    to full WENO, density / energy L1 of the routed form against FP64 after
    the same steps, max |div B| of both."""
    import numpy as np
    import torch
    import how_mhd as hm
    world, rank, local = dist_info()
    torch.cuda.set_device(local)
    n = args.n
    s = slice(3, n + 3)
    text = (f"nx {n}\nny {n}\nnz {n}\nnt 1\ntend 1000.0\ngam 1.6666666666666667\ncour 0.4\n"
            f"problem turb3d\nseed 12345\nx1bc periodic\nx2bc periodic\nx3bc periodic\n")
    out, ref = {}, None
    for name, prec, router in (("fp64", "fp64", "off"), ("mixed+learned", "mixed", "on")):
        p = hm.read_parameters(text + f"precision {prec}\nrouter {router}\n")
        with hm.Domain(p) as d:
            d.init_problem()
            stream = torch.cuda.ExternalStream(d.stream)
            t, _, _ = d.run(0.0, args.warmup)
            if router == "on":
                d.router_stats(reset=True)
            d.sync()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            t, steps, _ = d.run(t, args.turb_steps)
            e1.record(stream)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            q = d.get_state(0)
            b = d.get_face_b(0)
            st = d.router_stats() if router == "on" else None
        rho, en = q[0, s, s, s].copy(), q[7, s, s, s].copy()
        del q
        r = {"zone_cycles_per_s": n ** 3 * steps / (ms * 1e-3), "ms_per_step": ms / steps, "steps": steps,
             "t_end": t}
        r.update(div_report(b, n, p.dx))
        del b
        if st:
            r["full_weno_fraction"] = st[0] / max(st[0] + st[1], 1)
        if ref is None:
            ref = (rho, en)
        else:
            r["l1_rho_vs_fp64"] = float(np.abs(rho - ref[0]).sum() / np.abs(ref[0]).sum())
            r["l1_energy_vs_fp64"] = float(np.abs(en - ref[1]).sum() / np.abs(ref[1]).sum())
            r["speedup_vs_plain_fp64"] = r["zone_cycles_per_s"] / out["fp64"]["zone_cycles_per_s"]
        out[name] = r
    if rank == 0:
        print(json.dumps({"workload": f"decaying turbulence turb3d {n}^3 (seed 12345), {args.warmup} warm-up + "
                                      f"{args.turb_steps} timed steps from t = 0 per form",
                          "unit": UNIT, "timing": "CUDA events on the library's stream",
                          "forms": out}), flush=True)
    return 0


def ctypes_peak(hm):
    import ctypes
    v = ctypes.c_double()
    rc = hm.lib().how_measure_fp64_peak(ctypes.byref(v), 5)
    return v.value if rc == 0 else None


def main():
    args = parse()
    if args.n is None:
        args.n = 384 if args.workload == "turbulence" else 256
    if args.impl == "reference":
        return bench_reference(args)
    if args.workload == "ensemble":
        return bench_ensemble(args)
    if args.workload == "accuracy":
        return bench_accuracy(args)
    if args.workload == "output":
        return bench_output(args)
    if args.workload == "turbulence":
        return bench_turbulence(args)
    return bench_ours(args)


if __name__ == "__main__":
    sys.exit(main())
