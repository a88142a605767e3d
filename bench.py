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
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--t-start", type=float, default=0.05,
                    help="simulated time the timed steps start from (the blast evolved there first)")
    ap.add_argument("--no-fast", action="store_true", help="skip the mixed-precision + learned-routing leg")
    ap.add_argument("--workload", default="blast", choices=["blast", "ensemble", "accuracy", "output"],
                    help="ensemble: 64 uneven 2-D/1-D runs batched vs advanced one by one; "
                         "accuracy: whole blast run to --tend in every precision / routing form; "
                         "output: dump files (how_output) of the blast state, .vts and .dat")
    ap.add_argument("--out-dir", default="/tmp/how_dumps", help="--workload output: where the dumps go")
    ap.add_argument("--tend", type=float, default=0.2, help="end time of --workload accuracy")
    ap.add_argument("--forms", default="",
                    help="--workload accuracy: ';'-separated subset of the forms after fp64 (default: all)")
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


def run_reference_sample(steps, warmup, threads):
    """Time the reference's own CPU path (oracle/_ref/how_ref) on the 64^3 sample;
    returns (zone-cycles/s, kind, sample description).  Falls back to the oracle
    port (oracle/_build/liboracle.so) when the reference build is absent."""
    import numpy as np
    import how_mhd as hm
    n = REF_SAMPLE_N
    sample = (f"blast3d_b {n}^3 (the headline problem at a size the host finishes in seconds), "
              f"{steps} timed SSPRK step(s) after {warmup} warm-up, {threads} OpenMP threads")
    text = workload_text(n, "fp64")
    p = hm.read_parameters(text)
    q = hm.problem_state(p)
    binp = ref_binary()
    if binp is not None:
        sys.path.insert(0, str(REPO / "tests"))
        from howtest import write_dump
        with tempfile.TemporaryDirectory() as td:
            inp = Path(td) / "in.txt"
            inp.write_text(text)
            st = Path(td) / "state.bin"
            write_dump(st, {"q": q})
            env = dict(os.environ, OMP_NUM_THREADS=str(threads))
            r = subprocess.run([str(binp), str(inp), "/dev/null", "--state", str(st), "--steps", str(steps),
                                "--warmup", str(warmup), "--time-only", "--threads", str(threads)],
                               capture_output=True, text=True, env=env, timeout=3600)
            if r.returncode == 0:
                js = json.loads(r.stdout.strip().splitlines()[-1])
                return js["zone_cycles_per_s"], "reference", sample
    # oracle port
    sys.path.insert(0, str(REPO / "tests"))
    from howtest import CPUOracle, oracle_lib
    oracle_lib().oracle_set_threads(threads)
    o = CPUOracle(n, n, n, gam=5.0 / 3.0, rhomin=1e-6, pgmin=1e-6)
    o.set_state(q)
    for _ in range(warmup):
        o.ssprk(o.tstep())
    t0 = time.perf_counter()
    for _ in range(steps):
        o.ssprk(o.tstep())
    el = time.perf_counter() - t0
    return n ** 3 * steps / el, "port", sample.replace("OpenMP", "OpenMP (oracle port)")


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


# ---------------------------------------------------------------- reference arm
def bench_reference(args):
    world, rank, local = dist_info()
    if rank != 0:
        return 0
    threads = host_threads()
    t0 = time.perf_counter()
    zcs, kind, sample = run_reference_sample(max(args.steps, 1), args.warmup, threads)
    n3 = REF_SAMPLE_N ** 3
    line = {
        "impl": "reference", "metric": METRIC, "value": zcs, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * n3 / zcs,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": f"3-D MHD blast (blast3d_b) {REF_SAMPLE_N}^3 sample of the 256^3 workload, "
                               "reference Kokkos/OpenMP path built from its own sources"},
        "cpu_baseline": {"value": zcs, "unit": UNIT, "cores": threads, "kind": kind, "sample": sample},
        "e2e": {"value": zcs, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
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

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
        torch.cuda.synchronize()

    # The timed steps start from the blast at t_start (evolved by the fast path,
    # so every leg starts from the same mid-run state with a shock in the box).
    t0_prep = time.perf_counter()
    q_start = b_start = None
    t_start = 0.0
    if args.t_start > 0:
        pp = hm.read_parameters(workload_text(n, "mixed", tend=args.t_start, router="on"))
        with hm.Domain(pp) as d:
            d.init_problem()
            t_start, _, _ = d.run(0.0, -1)
            q_start = d.get_state(0)
            b_start = d.get_face_b(0)
    prep_s = time.perf_counter() - t0_prep

    def make_domain(precision, router):
        p = hm.read_parameters(workload_text(n, precision, router=router))
        dom = hm.Domain(p)
        if q_start is not None:
            dom.set_state(q_start)
            dom.set_face_b(*b_start)
        else:
            dom.init_problem()
        return p, dom

    def timed_leg(dom, clocks_too):
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
        e0.record(stream)
        dom.run(t_sim, args.steps)
        e1.record(stream)
        barrier()
        ms = e0.elapsed_time(e1)
        launches = dom.kernel_launches - l0
        sweep_ms = ctypes.c_double()
        sweep_n = ctypes.c_long()
        hm.lib().how_get_kernel_timing(dom._h, ctypes.byref(sweep_ms), ctypes.byref(sweep_n))
        hm.lib().how_set_kernel_timing(dom._h, 0)
        clocks = sampler.stop() if sampler else None
        return max_over_ranks(ms, world, "cuda"), launches, sweep_ms.value, sweep_n.value, clocks

    # ---- plain FP64 (the reference's method)
    p, dom = make_domain("fp64", "off")
    ms, launches, sweep_ms, sweep_n, clocks = timed_leg(dom, True)
    value = replica_value(world, n ** 3, args.steps, ms)
    rho64 = None
    if not args.no_fast and rank == 0:
        q64 = dom.get_state(0)
        rho64 = q64[0, 3:n + 3, 3:n + 3, 3:n + 3].copy()
        e64 = q64[7, 3:n + 3, 3:n + 3, 3:n + 3].copy()
        del q64

    # ---- e2e through the C ABI with pinned host buffers
    e2e = None
    if not args.no_e2e:
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

    # ---- mixed precision + learned routing (the fast form), same start, same steps
    fast = None
    if not args.no_fast:
        pf, domf = make_domain("mixed", "on")
        domf.router_stats(reset=True)
        fms, flaunch, fsw_ms, fsw_n, _ = timed_leg(domf, False)
        full, cheap = domf.router_stats()
        fvalue = replica_value(world, n ** 3, args.steps, fms)
        if rank == 0:
            qf = domf.get_state(0)
            bf = domf.get_face_b(0)
            rf = qf[0, 3:n + 3, 3:n + 3, 3:n + 3]
            ef = qf[7, 3:n + 3, 3:n + 3, 3:n + 3]
            w, thr = hm.default_router()
            fast = {
                "value": fvalue, "unit": UNIT, "ms_per_step": fms / args.steps,
                "speedup_vs_plain_fp64": fvalue / value,
                "full_weno_fraction": full / max(full + cheap, 1),
                "l1_rho_vs_fp64": float(np.abs(rf - rho64).sum() / np.abs(rho64).sum()),
                "l1_energy_vs_fp64": float(np.abs(ef - e64).sum() / np.abs(e64).sum()),
                "max_div_b": div4_max(bf, n, pf.dx),
                "router_threshold": thr, "gpu_launches": flaunch,
                "sweep_avg_ms": fsw_ms / max(fsw_n, 1),
                "note": "same start state and step count as the plain FP64 leg; L1 over active cells; the network decides once per step, the guard every stage",
            }
            del qf, bf
        domf.close()
        # the same form with the network's decisions formed at every stage
        pf, domf = make_domain("mixed", "on")
        domf.set_router_refresh(1)
        domf.router_stats(reset=True)
        sms, _, _, _, _ = timed_leg(domf, False)
        full5, cheap5 = domf.router_stats()
        if rank == 0:
            qf = domf.get_state(0)
            rf = qf[0, 3:n + 3, 3:n + 3, 3:n + 3]
            v5 = replica_value(world, n ** 3, args.steps, sms)
            fast["decisions_every_stage"] = {
                "value": v5, "ms_per_step": sms / args.steps, "speedup_vs_plain_fp64": v5 / value,
                "full_weno_fraction": full5 / max(full5 + cheap5, 1),
                "l1_rho_vs_fp64": float(np.abs(rf - rho64).sum() / np.abs(rho64).sum()),
            }
            del qf
        domf.close()

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
        threads = host_threads()
        zcs, kind, sample = run_reference_sample(1, 1, threads)
        cpu = {"value": zcs, "unit": UNIT, "cores": threads, "kind": kind, "sample": sample}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": f"3-D MHD blast {n}^3 (blast3d_b), periodic, gam 5/3, cour 0.4, floors 1e-6; "
                               f"SSPRK(5,4) + characteristic WENO5/LLF + 4th-order CT; `value` = plain FP64, "
                               f"`mixed_learned` = FP32 characteristic part + learned WENO routing",
                   "n": n, "t_start": t_start, "prep_s": prep_s,
                   "parallelism": "replicas" if world > 1 else "single",
                   "l2": "state 12.5 GB per replica >> 126 MB L2: every step streams from HBM, no flush"},
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
    with hm.Ensemble(members) as e:
        e.init()
        e.run(args.warmup + 3)               # autotune (3 steps) + warm-up
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e.run(args.steps)
        torch.cuda.synchronize()
        ens_s = time.perf_counter() - t0
        shapes, sweep_ms = e.shapes()
        launches = e.graph_launches
    # one by one, same K steps per member (each with its own warm-up)
    seq_s = 0.0
    for p in members:
        with hm.Domain(p) as d:
            d.init_problem()
            t, _, _ = d.run(0.0, args.warmup)
            d.sync()
            t0 = time.perf_counter()
            d.run(t, args.steps)
            d.sync()
            seq_s += time.perf_counter() - t0
    if rank != 0:
        return 0
    value = world * zones * args.steps / ens_s
    line = {
        "metric": "zone-cycles/s, batched ensemble of 64 uneven 2-D/1-D runs, 1 B200", "value": value,
        "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * ens_s / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "24 Orszag-Tang + 24 MHD rotors at {64..512}^2, 16 Brio-Wu at nx {400,800,1600}",
                   "members": len(members), "zones": zones, "timing": "host clock around synchronised runs"},
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


def ctypes_peak(hm):
    import ctypes
    v = ctypes.c_double()
    rc = hm.lib().how_measure_fp64_peak(ctypes.byref(v), 5)
    return v.value if rc == 0 else None


def main():
    args = parse()
    if args.impl == "reference":
        return bench_reference(args)
    if args.workload == "ensemble":
        return bench_ensemble(args)
    if args.workload == "accuracy":
        return bench_accuracy(args)
    if args.workload == "output":
        return bench_output(args)
    return bench_ours(args)


if __name__ == "__main__":
    sys.exit(main())
