#!/usr/bin/env python
"""HOLD step throughput on B200: top-level HOLD steps/s and pair interactions/s.

Workload (one GPU): a seeded Plummer sphere, N = 16384 equal masses, Henon units,
eta = 0.03, top-level step dt = 2^-6, mixed precision (FP32 pair terms, FP64 state).
A "step" is one top-level hold_step (timesteps recomputed at the top). Inputs are
resident in HBM when the timed region starts; L2 is flushed between timed steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU: a single system does not shard (replicas only): each rank integrates its
own independently seeded sphere; value = all ranks' steps / max-over-ranks time.
--impl reference times the CPU FP64 restatement of the reference HOLD step (the
reference has no CPU HOLD of its own) on the host cores, on rank 0 only.
"""
import argparse
import ctypes
import json
import os
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "parallel-hhs_b200"))

METRIC = "pair interactions/s & HOLD steps/s at |dE/E|<=1e-6 vs plain FP64 GPU path"
KICK_FLOPS_PER_PAIR = 20.0   # conventional direct-sum count (Nyland, Harris & Prins 2007)
L2_FLUSH_BYTES = 256 << 20


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--n", type=int, default=16384)
    p.add_argument("--eta", type=float, default=0.03)
    p.add_argument("--dt", type=float, default=2.0 ** -6)
    p.add_argument("--seed", type=int, default=2024)
    p.add_argument("--prec", default="mixed", choices=["mixed", "fp64"])
    p.add_argument("--schedule", default="auto", choices=["auto", "host"])
    p.add_argument("--small-n", type=int, default=64,
                   help="device schedule: nodes with n <= this are solved by one CTA")
    p.add_argument("--ctas-per-sm", type=int, default=2)
    p.add_argument("--cluster-size", type=int, default=4,
                   help="launch the HOLD kernel in thread-block clusters of this size")
    p.add_argument("--mid-n", type=int, default=640,
                   help="subtrees of at most this many particles run from shared memory on "
                        "one cluster (0 = off)")
    p.add_argument("--mid-dist-n", type=int, default=96,
                   help="inside such a subtree, nodes above this size spread over the cluster")
    p.add_argument("--packed", type=int, default=0)
    p.add_argument("--overlap", type=int, default=1,
                   help="slow-only kick units beside a subtree's first pass (1) or not (0)")
    p.add_argument("--units-per-cta", type=int, default=16)
    p.add_argument("--no-autotune", dest="autotune", action="store_false",
                   help="keep the given tuning instead of the library's autotuner's pick")
    p.add_argument("--profile-out", default=None,
                   help="write the per-level phase profile (JSON) to this path")
    p.add_argument("--workload", default="plummer16k",
                   choices=["plummer16k", "batched", "scan", "large", "deep", "validate",
                            "plain1k", "kickprobe", "tsprobe"],
                   help="plummer16k (default headline), batched (512 clusters), scan (flag "
                        "compaction sweep), large (N=262144, 90/10 masses), deep (N=65536 "
                        "Salpeter), validate (integrate --n/--eta/--mass to --t-end in mixed "
                        "and FP64 precision and compare), plain1k (N=1024 FP64 to t=1 on the "
                        "GPU and on the CPU oracle, compared bit for bit)")
    p.add_argument("--t-end", type=float, default=1.0)
    p.add_argument("--mass", type=int, default=0, choices=[0, 1, 2],
                   help="mass spectrum: 0 equal, 1 Salpeter on [0.1, 100], 2 90%%/10%% two-component")
    p.add_argument("--scan-log2n", type=int, default=None,
                   help="scan workload: run this one size instead of the 2^20..2^28 sweep")
    p.add_argument("--no-baselines", action="store_true",
                   help="skip the FP64 GPU and CPU baselines (quick runs)")
    return p.parse_args()


MASS_NAMES = {0: "equal-mass", 1: "Salpeter dN/dm ~ m^-2.35 on [0.1,100]",
              2: "two-component (90% m=1, 10% m=10)"}


def workload_name(a):
    return (f"Plummer N={a.n} {MASS_NAMES[getattr(a, 'mass', 0)]}, Henon units, eta={a.eta}, "
            f"dt_top=2^{int(round(__import__('math').log2(a.dt)))}, "
            f"one top-level HOLD step per step")


# ------------------------------------------------------------------------ ranks
def replica_seed(seed, rank):
    """Each rank integrates its own independently seeded system (replicas only)."""
    return seed + 7919 * rank


def max_over_ranks(value, dist, torch, device="cuda"):
    """Max over all ranks of a per-rank time (the job's time is its slowest rank)."""
    if dist is None:
        return value
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def cluster_sizes(seed, count=512, lo=64, hi=4096):
    """Cluster sizes of the batched workload: log-uniform in [lo, hi] from the seed."""
    import numpy as np
    rng = np.random.default_rng(seed)
    return np.round(np.exp(rng.uniform(np.log(lo), np.log(hi), count))).astype(np.int64)


def gather_by_index(local_idx, local_vals, n_total, dist):
    """Reassembles per-cluster values computed on the ranks (each rank holds the values of
    the clusters local_idx) into one array in cluster order; the batched workload's only
    collective, taken once after the timed region."""
    import numpy as np
    out = np.full(n_total, np.nan)
    if dist is None:
        out[np.asarray(local_idx)] = local_vals
        return out
    parts = [None] * dist.get_world_size()
    dist.all_gather_object(parts, (list(map(int, local_idx)), list(map(float, local_vals))))
    for idx, vals in parts:
        out[np.asarray(idx, dtype=np.int64)] = vals
    return out


def aggregate_value(steps, world, t_max_ms):
    """Whole-job throughput: all ranks' steps over the max-over-ranks time."""
    return steps * world / (t_max_ms * 1e-3)


# ------------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi clock and throttle-reason samples every 50 ms on a reader thread; only
    the samples taken between mark_start() and mark_stop() (the timed region) count."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, dev):
        self.dev = dev
        self.p = None
        self.lines = []
        self.t0 = self.t1 = None
        self.th = None

    def start(self):
        import threading
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "50",
                                       "-i", str(self.dev)], stdout=subprocess.PIPE,
                                      stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.p = None
            return

        def reader():
            for line in self.p.stdout:
                self.lines.append((time.monotonic(), line))

        self.th = threading.Thread(target=reader, daemon=True)
        self.th.start()
        deadline = time.monotonic() + 5.0
        while not self.lines and time.monotonic() < deadline:
            time.sleep(0.01)

    def mark_start(self):
        self.t0 = time.monotonic()

    def mark_stop(self):
        self.t1 = time.monotonic()
        # let the sampler take at least one more sample past the region's end
        time.sleep(0.06)

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        if self.th is not None:
            self.th.join(timeout=5)
        inside = [l for t, l in self.lines
                  if self.t0 is not None and self.t1 is not None and self.t0 <= t <= self.t1 + 0.06]
        use = inside if inside else [l for _, l in self.lines]
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in use:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        if not sm:
            return None
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm), "in_timed_region": bool(inside)}


# ------------------------------------------------------------------------ reference arm
def mapped_libraries():
    """Shared objects mapped into this process (from /proc/self/maps)."""
    out = set()
    try:
        with open("/proc/self/maps") as f:
            for line in f:
                parts = line.split()
                if len(parts) >= 6 and (parts[-1].endswith(".so") or ".so." in parts[-1]):
                    out.add(parts[-1])
    except OSError:
        pass
    return sorted(out)


def run_reference(a, rank, world, isolated=True):
    """CPU FP64 restatement of the reference HOLD step on the host cores (rank 0). The
    initial conditions come from the oracle's own generator (the same arrays as the
    product's), so with isolated=True (the --impl reference process) nothing of the
    product library is loaded; that is checked before the timed loop."""
    if rank != 0:
        return None
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    oracle.build()
    s = oracle.plummer(a.n, a.seed, getattr(a, "mass", 0))
    if isolated:
        product = [m for m in mapped_libraries() if "libhhs_b200" in m]
        if product:
            raise RuntimeError(f"reference arm has the product library mapped: {product}")
    budget_s = 150.0
    t0 = time.perf_counter()
    oracle.hold_step(s, a.dt, True, a.eta)           # warm-up steps, as many as asked for
    one = time.perf_counter() - t0                   # within a quarter of the budget
    warm = 1
    while warm < getattr(a, "warmup", 1) and (warm + 1) * one < 0.25 * budget_s:
        oracle.hold_step(s, a.dt, True, a.eta)
        warm += 1
    steps = max(1, min(a.steps, int(budget_s / max(one, 1e-3))))
    t0 = time.perf_counter()
    for _ in range(steps):
        oracle.hold_step(s, a.dt, True, a.eta)
    el = time.perf_counter() - t0
    v = steps / el
    cores = oracle.threads()
    out = {"metric": METRIC, "value": v, "unit": "HOLD steps/s", "impl": "reference",
           "n_gpus": world, "steps": steps, "warmup": warm, "ms_per_step": el / steps * 1e3,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic", "config": {"workload": workload_name(a), "n": a.n, "eta": a.eta,
                                            "dt_top": a.dt, "precision": "fp64 (CPU oracle)"},
           "cpu_baseline": {"value": v, "unit": "HOLD steps/s", "cores": cores, "kind": "port",
                            "sample": f"{steps} top-level HOLD step(s) of the same N={a.n} "
                                      f"Plummer sphere, FP64 CPU restatement, OpenMP "
                                      f"{cores} threads (the reference has no CPU HOLD)"},
           "e2e": {"value": v, "unit": "HOLD steps/s", "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0}}
    if isolated:
        out["libraries_mapped"] = [m for m in mapped_libraries() if ROOT in m]
    return out


# ------------------------------------------------------------------------ our arm
def run_ours(a, rank, world, torch, dist):
    import numpy as np
    import hhs

    dev = torch.cuda.current_device()
    stream = torch.cuda.Stream()
    sh = ctypes.c_void_p(stream.cuda_stream)
    prec = hhs.PREC_MIXED if a.prec == "mixed" else hhs.PREC_FP64
    seed = replica_seed(a.seed, rank)
    ics = hhs.plummer(a.n, seed, getattr(a, "mass", 0))
    e0 = hhs.energy_host(ics)
    ctx = hhs.Context(a.n, 64, eta=a.eta)
    ctx.set_tuning(a.small_n, a.units_per_cta, a.ctas_per_sm, cluster_size=a.cluster_size,
                   mid_n=a.mid_n, packed=a.packed, mid_dist_n=a.mid_dist_n, overlap=a.overlap)
    sys_ = hhs.ParticleSystem(a.n)
    sys_.upload(ics, stream=sh)
    tuned = None
    if a.autotune and a.schedule == "auto":
        tuned = {"chosen": ctx.autotune(sys_, a.n, a.dt, prec, stream=sh),
                 "candidates": ctx.autotune_results()}
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")

    def step(p=prec):
        if a.schedule == "host":
            hhs.hold_step_host(ctx, sys_, a.n, a.dt, True, p, stream=sh)
        else:
            hhs.hold_step(ctx, sys_, a.n, 0.0, a.dt, True, p, stream=sh)

    def barrier():
        if dist is not None:
            dist.barrier()

    with torch.cuda.stream(stream):
        for _ in range(a.warmup):
            step()
        ctx.check(sh)
        ctx.reset_stats(sh)
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(a.steps)]
        clocks = ClockSampler(dev)
        barrier()
        torch.cuda.synchronize()
        clocks.start()
        clocks.mark_start()
        l0 = hhs.launch_count()
        for k in range(a.steps):
            flush.zero_()
            evs[k][0].record(stream)
            step()
            evs[k][1].record(stream)
        torch.cuda.synchronize()
        l1 = hhs.launch_count()
        clocks.mark_stop()
        barrier()
        clk = clocks.stop()
        ctx.check(sh)
        t_ms = sum(e0_.elapsed_time(e1_) for e0_, e1_ in evs)
        stats = ctx.stats(sh)
        out = sys_.download(stream=sh)
        torch.cuda.synchronize()
        # the phase profile (timer reads at every phase boundary) from separate steps after
        # the timed ones, so that it does not weigh on the timed region
        ctx.reset_stats(sh)
        ctx.set_profiling(True)
        prof_steps = min(a.steps, 5)
        for _ in range(prof_steps):
            step()
        torch.cuda.synchronize()
        ctx.check(sh)
        prof = {k: dict(v, launches=v["launches"] * a.steps // prof_steps,
                        ms=v["ms"] * a.steps / prof_steps,
                        pairs=v["pairs"] * a.steps / prof_steps)
                for k, v in ctx.profile().items()}
        if a.profile_out and a.schedule == "auto":
            lms, lcnt = ctx.level_profile()
            kinds = ["timesteps", "kick", "split", "update", "engine", "subtree", "cluster_node",
                     "subtree_stages"]
            lp = {kinds[k]: {str(l): [round(float(lms[k, l]) / prof_steps, 4),
                                      int(lcnt[k, l]) // prof_steps]
                             for l in range(64) if lcnt[k, l]} for k in range(8)}
            with open(a.profile_out, "w") as f:
                json.dump({"per_step_ms_and_phases_by_level": lp, "tuning": ctx.tuning()}, f,
                          indent=1)
        ctx.set_profiling(False)
    e1 = hhs.energy_host(out)

    t_max = max_over_ranks(t_ms, dist, torch)
    steps_total = a.steps * world
    value = aggregate_value(a.steps, world, t_max)
    pairs_step = (stats["kick_pairs"] + stats["ts_pairs"]) / a.steps
    res = {"value": value, "t_ms": t_max, "pairs_per_step": pairs_step, "stats": stats,
           "tuning": ctx.tuning(), "autotune": tuned,
           "prof": prof, "clocks": clk, "launches": (l1 - l0), "dE_over_E": (e1 - e0) / e0}

    # ---- end to end through the public API: host buffers, copies inside the timed region
    pin = {k: torch.from_numpy(np.ascontiguousarray(out[k])).pin_memory().numpy()
           for k in ("x", "y", "z", "vx", "vy", "vz", "m", "ts")}
    pin["id"] = torch.from_numpy(out["id"].copy()).pin_memory().numpy()
    res_pin = {k: torch.empty(a.n, dtype=torch.float64).pin_memory().numpy()
               for k in ("x", "y", "z", "vx", "vy", "vz", "ts")}
    h2d = a.n * (8 * 8 + 4)
    d2h = a.n * 7 * 8
    L = hhs.lib()
    dp = ctypes.POINTER(ctypes.c_double)
    ip = ctypes.POINTER(ctypes.c_int32)

    def pp(arr, t=dp):
        return None if arr is None else arr.ctypes.data_as(t)

    with torch.cuda.stream(stream):
        e2e_ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                  for _ in range(a.steps)]
        barrier()
        torch.cuda.synchronize()
        for k in range(a.steps):
            flush.zero_()
            e2e_ev[k][0].record(stream)
            assert L.hhs_particle_system_upload(sys_.ref, a.n, *[pp(pin[f]) for f in
                                                                 ("x", "y", "z", "vx", "vy", "vz",
                                                                  "m", "ts")],
                                                pp(pin["id"], ip), sh) == 0
            step()
            assert L.hhs_particle_system_download(sys_.ref, a.n, *[pp(res_pin.get(f)) for f in
                                                                   ("x", "y", "z", "vx", "vy",
                                                                    "vz", "m", "ts")],
                                                  None, sh) == 0
            e2e_ev[k][1].record(stream)
            stream.synchronize()
            for f in res_pin:
                pin[f][:] = res_pin[f]
        torch.cuda.synchronize()
        barrier()
    t_e2e = max_over_ranks(sum(x.elapsed_time(y) for x, y in e2e_ev), dist, torch)
    res["e2e"] = {"value": steps_total / (t_e2e * 1e-3), "unit": "HOLD steps/s",
                  "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h}

    # ---- plain FP64 GPU HOLD (host-driven schedule): the denominator of the target
    if not a.no_baselines:
        k64 = max(2, a.steps // 5)
        sys64 = hhs.ParticleSystem(a.n)
        sys64.upload(ics, stream=sh)
        with torch.cuda.stream(stream):
            hhs.hold_step_host(ctx, sys64, a.n, a.dt, True, hhs.PREC_FP64, stream=sh)
            evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                   for _ in range(k64)]
            torch.cuda.synchronize()
            for k in range(k64):
                flush.zero_()
                evs[k][0].record(stream)
                hhs.hold_step_host(ctx, sys64, a.n, a.dt, True, hhs.PREC_FP64, stream=sh)
                evs[k][1].record(stream)
            torch.cuda.synchronize()
        t64 = sum(x.elapsed_time(y) for x, y in evs)
        res["fp64_plain_steps_per_s"] = k64 / (t64 * 1e-3)
        res["fp64_plain_steps"] = k64
        # the same FP64 kernels' arithmetic on the device-resident schedule (information)
        if a.schedule == "auto":
            with torch.cuda.stream(stream):
                hhs.hold_step(ctx, sys64, a.n, 0.0, a.dt, True, hhs.PREC_FP64, stream=sh)
                torch.cuda.synchronize()
                for k in range(k64):
                    flush.zero_()
                    evs[k][0].record(stream)
                    hhs.hold_step(ctx, sys64, a.n, 0.0, a.dt, True, hhs.PREC_FP64, stream=sh)
                    evs[k][1].record(stream)
                torch.cuda.synchronize()
                ctx.check(sh)
            res["fp64_engine_steps_per_s"] = k64 / (sum(x.elapsed_time(y) for x, y in evs) * 1e-3)
    res["fma_peaks"] = hhs.measure_fma_peaks(sh)
    res["fma2_peak"] = hhs.measure_fma2_peak(sh)
    return res


# DRAM bytes of one k_engine launch of the default workload (dram__bytes_read.sum +
# dram__bytes_write.sum of an ncu capture of one launch after three warm-up launches)
ENGINE_16K_DRAM_BYTES = 1.582336e6 + 2.816000e6


def nominal_fp32_tflops(torch):
    """Nominal FP32 FMA peak of the device: SMs x 128 FP32 lanes x 2 flops x max SM clock
    (nvidia-smi clocks.max.sm; 1965 MHz on B200 when it cannot be read)."""
    sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    mhz = 1965.0
    try:
        q = subprocess.run(["nvidia-smi", "--query-gpu=clocks.max.sm", "--format=csv,noheader,nounits",
                            "-i", str(torch.cuda.current_device())], capture_output=True,
                           text=True, timeout=20)
        mhz = float(q.stdout.strip().splitlines()[0])
    except (OSError, ValueError, IndexError, subprocess.SubprocessError):
        pass
    return sms * 128 * 2 * mhz * 1e6 / 1e12


def roofline(res, a, peaks_tflops, nominal_tflops):
    """Roofline of the dominant kernel, the persistent HOLD kernel (one launch per step),
    counted as the kick work alone: kick pairs (N_s(N_s-1) + 2 N_s N_f per node, from the
    run's own work counters) x 20 flops over the launch's CUDA-event duration. Timestep
    pair evaluations are reported beside it as a rate, with no flop credit. The peak is
    the measured FP32 FMA-chain rate of this B200; the nominal FP32 peak is given too."""
    prof = res["prof"]
    st = res["stats"]
    launch_ms = res["t_ms"] / a.steps
    flops = st["kick_pairs"] * KICK_FLOPS_PER_PAIR / a.steps
    achieved = flops / (launch_ms * 1e-3) / 1e12
    peak = peaks_tflops[0] if a.prec == "mixed" else peaks_tflops[1]
    phases = {}
    for kind in ("timesteps", "kick", "split", "update", "cluster_node", "subtree"):
        p = (prof or {}).get(kind)
        if p and p["ms"] > 0:
            phases[kind] = {"ms_per_step": p["ms"] / a.steps, "share_of_step": p["ms"] / res["t_ms"]}
    kp = (prof or {}).get("kick")
    if kp and kp["ms"] > 0:
        tf = kp["pairs"] * KICK_FLOPS_PER_PAIR / (kp["ms"] * 1e-3) / 1e12
        phases["kick"].update({"achieved": tf, "frac": tf / peak})
    tp = (prof or {}).get("timesteps")
    if tp and tp["ms"] > 0:
        phases["timesteps"]["unordered_pair_evaluations_per_s"] = tp["pairs"] / 2 / (tp["ms"] * 1e-3)
    default = (a.n == 16384 and a.prec == "mixed" and a.workload == "plummer16k")
    out = {"bound": "fp32-fma" if a.prec == "mixed" else "fp64-fma", "kernel": "k_engine",
           "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
           "peak_source": "measured FMA-chain peak of this B200 (hhs_measure_fma_peaks); "
                          "the pair kernels use neither tensor cores nor HBM bandwidth",
           "flops_per_launch": flops, "flops_per_pair": KICK_FLOPS_PER_PAIR,
           "work": "kick pairs x 20 flops (timestep work not counted)",
           "launch_ms": launch_ms, "phases": phases,
           "traffic": ENGINE_16K_DRAM_BYTES if default else None,
           "traffic_note": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch "
                           "of this workload" if default else None}
    if a.prec == "mixed":
        out["peak_nominal"] = nominal_tflops
        out["frac_of_nominal"] = achieved / nominal_tflops
    return out


# ------------------------------------------------------------------------ other workloads
def run_batched(a, torch, rank=0, world=1, dist=None):
    """512 independent Plummer clusters, N log-uniform in [64, 4096], one launch per step.
    With several ranks the clusters are sharded by hhs_batch_partition (balanced sum of
    N^2, no data exchange); value = all clusters' steps over the max-over-ranks time."""
    import numpy as np
    import hhs
    sizes = cluster_sizes(a.seed)
    mine = hhs.batch_shard(sizes, world, rank) if world > 1 else np.arange(len(sizes))
    parts = [hhs.plummer(int(sizes[k]), a.seed * 1000 + int(k)) for k in mine]
    e0 = np.array([hhs.energy_host(p) for p in parts])
    packed = {f: np.concatenate([p[f] for p in parts]) for f in hhs.FIELDS}
    n = int(sum(len(p["x"]) for p in parts))
    packed["id"] = np.arange(n, dtype=np.int32)
    off = np.concatenate([[0], np.cumsum([len(p["x"]) for p in parts])]).astype(np.int32)
    stream = torch.cuda.Stream()
    sh = ctypes.c_void_p(stream.cuda_stream)
    prec = hhs.PREC_MIXED if a.prec == "mixed" else hhs.PREC_FP64
    d = hhs.ParticleSystem(n)
    d.upload(packed, stream=sh)
    b = hhs.Batch(off, 64, eta=a.eta)
    tuned = None
    if getattr(a, "autotune", True):
        best, table = b.autotune(d, a.dt, prec, stream=sh)
        tuned = {"chosen": best, "candidates": table}
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")
    with torch.cuda.stream(stream):
        for _ in range(a.warmup):
            b.step(d, a.dt, True, prec, stream=sh)
        b.check(sh)
        b.reset_stats(sh)
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(a.steps)]
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        for k in range(a.steps):
            flush.zero_()
            evs[k][0].record(stream)
            b.step(d, a.dt, True, prec, stream=sh)
            evs[k][1].record(stream)
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        b.check(sh)
    t_ms = max_over_ranks(sum(x.elapsed_time(y) for x, y in evs), dist, torch)
    st = b.stats(sh)
    pairs = st["kick_pairs"] + st["ts_pairs"]
    if dist is not None:
        tp = torch.tensor([pairs], dtype=torch.float64, device="cuda")
        dist.all_reduce(tp)
        pairs = float(tp.item())
    out = d.download()
    de = []
    for k in range(len(parts)):
        sl = slice(off[k], off[k + 1])
        e1 = hhs.energy_host({f: np.ascontiguousarray(out[f][sl]) for f in ("x", "y", "z", "vx",
                                                                            "vy", "vz", "m")})
        de.append(abs((e1 - e0[k]) / e0[k]))
    de = gather_by_index(mine, de, len(sizes), dist)
    steps_all = a.steps + a.warmup
    n_total = int(sizes.sum())
    return {"metric": "aggregate HOLD steps/s over 512 independent clusters",
            "value": len(sizes) * a.steps / (t_ms * 1e-3), "unit": "cluster HOLD steps/s",
            "launches_per_s": a.steps / (t_ms * 1e-3), "ms_per_step": t_ms / a.steps,
            "steps": a.steps, "warmup": a.warmup, "n_gpus": world, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None,
            "dtype": "f32-pair/f64-state" if a.prec == "mixed" else "f64",
            "data": "synthetic (seeded Plummer clusters)",
            "config": {"workload": f"512 Plummer clusters, N log-uniform [64,4096] "
                                   f"(total {n_total}), eta={a.eta}, dt_top={a.dt}, one launch "
                                   f"per top step per rank",
                       "n_total": n_total, "l2": "flushed between timed steps",
                       "autotuned": tuned is not None, "autotune": tuned,
                       "parallelism": f"clusters sharded x{world} (balanced sum N^2)"},
            "pair_interactions_per_s": pairs / (t_ms * 1e-3),
            "dE_over_E_after_steps": {"steps": steps_all, "median": float(np.median(de)),
                                      "p90": float(np.percentile(de, 90)),
                                      "max": float(de.max())}}


def ref_scan_in_bounds(n, bs, unroll=4):
    """True when the reference's scan recursion (src/split.cuh:438-565) never calls
    scan_predicate_small with fewer than 3 elements, which writes past its dynamic
    shared buffer; only such sizes are run."""
    e = bs * unroll
    calls = []

    def large(m):
        rem = m % e
        large_ev(m - rem)
        if rem:
            calls.append(rem)

    def large_ev(m):
        nb = (m + e - 1) // e
        (large if nb > e else calls.append)(nb)

    (large if n > e else calls.append)(n)
    return all(m >= 3 for m in calls)


def run_scan(a, torch):
    """Exclusive scan and stream compaction of Bernoulli(p) int32 flags, 2^20 .. 2^28."""
    import hhs
    ref = None
    ref_path = os.path.join(ROOT, "oracle", "_ref", "libref_gpu_nofma.so")
    if os.path.exists(ref_path):
        ref = ctypes.CDLL(ref_path)
        ref.ref_scan_predicate.argtypes = [ctypes.c_void_p] * 2 + [ctypes.c_int] * 2
    stream = torch.cuda.current_stream()
    sh = ctypes.c_void_p(stream.cuda_stream)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")
    rows = []

    def ptr(t):
        return ctypes.c_void_p(t.data_ptr())

    def timed(fn, reps):
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(reps)]
        fn()
        torch.cuda.synchronize()
        for k in range(reps):
            flush.zero_()
            ev[k][0].record()
            fn()
            ev[k][1].record()
        torch.cuda.synchronize()
        return sum(x.elapsed_time(y) for x, y in ev) / reps

    sizes = [a.scan_log2n] if a.scan_log2n else list(range(20, 29, 2))
    probs = (0.5,) if a.scan_log2n else (0.01, 0.1, 0.5)
    for lg in sizes:
        n = 1 << lg
        ws_b = hhs.scan_workspace_size(n)
        ws = torch.empty(ws_b, dtype=torch.uint8, device="cuda")
        out = torch.empty(n, dtype=torch.int32, device="cuda")
        idx = torch.empty(n, dtype=torch.int32, device="cuda")
        cnt = torch.zeros(1, dtype=torch.int32, device="cuda")
        for p in probs:
            g = torch.Generator(device="cuda").manual_seed(lg * 10 + int(p * 100))
            flags = (torch.rand(n, device="cuda", generator=g) < p).to(torch.int32)
            ms_scan = timed(lambda: hhs.scan_exclusive_i32(ptr(flags), ptr(out), n, ptr(ws), ws_b,
                                                           sh), a.steps)
            ok = bool(torch.equal(out[1:] - out[:-1], flags[:-1])) and int(out[0]) == 0
            ms_comp = timed(lambda: hhs.compact_flags_i32(ptr(flags), None, ptr(idx), ptr(cnt), n,
                                                          ptr(ws), ws_b, sh), a.steps)
            k = int(cnt.item())
            row = {"log2n": lg, "p": p, "scan_ms": ms_scan, "scan_GBps": 8 * n / ms_scan / 1e6,
                   "compact_ms": ms_comp, "compact_GBps": (4 * n + 4 * k) / ms_comp / 1e6,
                   "scan_properties_ok": ok, "selected": k}
            bs = next((b for b in (256, 128) if ref_scan_in_bounds(n, b)), None)
            if ref is not None and bs is not None:
                rout = torch.empty_like(flags)
                ms_ref = timed(lambda: ref.ref_scan_predicate(ptr(flags), ptr(rout), n, bs), 3)
                row["reference_scan_ms"] = ms_ref
                row["reference_scan_GBps"] = 8 * n / ms_ref / 1e6
                row["bit_exact_vs_reference"] = bool(torch.equal(rout, out))
            rows.append(row)
        del ws, out, idx, flags
        torch.cuda.empty_cache()
    top = [r for r in rows if r["log2n"] == sizes[-1] and r["p"] == 0.5][0]
    return {"metric": f"exclusive scan HBM GB/s (8 B/element), 2^{sizes[-1]} int32 flags, p=0.5",
            "value": top["scan_GBps"], "unit": "GB/s", "n_gpus": 1, "steps": a.steps,
            "higher_is_better": True, "dtype": "i32", "data": "synthetic Bernoulli flags",
            "config": {"workload": "scan/compaction sweep 2^20..2^28, p in {0.01,0.1,0.5}",
                       "l2": "flushed between timed calls"},
            "roofline": {"bound": "hbm", "achieved": top["scan_GBps"],
                         "unit": "GB/s", "traffic": None}, "sweep": rows}


def run_kickprobe(a, torch):
    """The engine's mixed kick phase alone (hhs_engine_kick_accelerations: a split node
    with every third particle fast) on a seeded sphere of --n particles: kick pairs per
    second (2 N_f N_s + N_s (N_s - 1) ordered sink-source pairs per call, the count of
    the reference's kick_sf + kick_slow), and the same as FP32 FLOP/s at 20 flops a pair."""
    import hhs
    n = a.n
    s = hhs.plummer(n, a.seed)
    ctx = hhs.Context(n, 64, eta=a.eta)
    d = hhs.ParticleSystem(n)
    d.upload(s)
    L = hhs.lib()
    for _ in range(a.warmup):
        assert L.hhs_engine_kick_accelerations(ctx.h, d.ref, n, None) == 0
    ctx.check()
    ev = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
    torch.cuda.synchronize()
    ev[0].record()
    for _ in range(a.steps):
        assert L.hhs_engine_kick_accelerations(ctx.h, d.ref, n, None) == 0
    ev[1].record()
    ctx.check()
    ms = ev[0].elapsed_time(ev[1]) / a.steps
    nf = (n + 2) // 3
    ns = n - nf
    pairs = 2 * nf * ns + ns * (ns - 1)
    return {"metric": "engine kick pairs/s", "value": pairs / (ms * 1e-3),
            "unit": "kick pairs/s", "n": n, "n_fast": nf, "n_slow": ns, "ms": ms,
            "tflops_at_20_per_pair": 20.0 * pairs / (ms * 1e-3) * 1e-12}


def run_tsprobe(a, torch):
    """The engine's mixed timestep phase alone (hhs_engine_timestep_rates: one node of --n
    particles, packed symmetric tiles) on a seeded sphere: unordered pair evaluations per
    second (n (n - 1) / 2 per call; each gives the pair's rate to both particles)."""
    import hhs
    n = a.n
    s = hhs.plummer(n, a.seed)
    ctx = hhs.Context(n, 64, eta=a.eta)
    d = hhs.ParticleSystem(n)
    d.upload(s)
    L = hhs.lib()
    for _ in range(a.warmup):
        assert L.hhs_engine_timestep_rates(ctx.h, d.ref, n, None) == 0
    ctx.check()
    ev = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
    torch.cuda.synchronize()
    ev[0].record()
    for _ in range(a.steps):
        assert L.hhs_engine_timestep_rates(ctx.h, d.ref, n, None) == 0
    ev[1].record()
    ctx.check()
    ms = ev[0].elapsed_time(ev[1]) / a.steps
    pairs = n * (n - 1) // 2
    return {"metric": "engine timestep unordered pairs/s", "value": pairs / (ms * 1e-3),
            "unit": "pair evaluations/s", "n": n, "ms": ms}


def run_plain1k(a, torch):
    """Plain FP64 HOLD of a Plummer N=1024 sphere to t=1 on the GPU (device schedule) and on
    the CPU oracle (OpenMP, host cores): the final states must agree bit for bit."""
    import numpy as np
    import hhs
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    oracle.build()
    n, eta, dt = 1024, 0.03, a.dt
    steps = int(round(1.0 / dt))
    ics = hhs.plummer(n, a.seed)
    e0 = hhs.energy_host(ics)
    ctx = hhs.Context(n, 64, eta=eta)
    d = hhs.ParticleSystem(n)
    d.upload(ics)
    ev = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
    torch.cuda.synchronize()
    ev[0].record()
    for _ in range(steps):
        hhs.hold_step(ctx, d, n, 0.0, dt, True, hhs.PREC_FP64)
    ev[1].record()
    ctx.check()
    gpu = d.download()
    t_gpu = ev[0].elapsed_time(ev[1]) * 1e-3
    ref = {k: v.copy() for k, v in ics.items()}
    t0 = time.perf_counter()
    for _ in range(steps):
        oracle.hold_step(ref, dt, True, eta)
    t_cpu = time.perf_counter() - t0
    same = all(np.array_equal(gpu[k], ref[k]) for k in hhs.FIELDS)
    return {"metric": "plain FP64 HOLD, Plummer N=1024 to t=1: GPU vs CPU oracle",
            "value": steps / t_gpu, "unit": "HOLD steps/s", "n": n, "eta": eta, "dt_top": dt,
            "steps": steps, "gpu_steps_per_s": steps / t_gpu,
            "cpu_oracle_steps_per_s": steps / t_cpu, "cpu_threads": oracle.threads(),
            "bit_exact_gpu_vs_oracle": bool(same),
            "dE_over_E": (hhs.energy_host(gpu) - e0) / e0}


def run_validate(a, torch, tuning=None):
    """Integrates the workload to t_end in mixed precision and in FP64 (the FP64 device
    schedule reproduces the CPU oracle bit for bit) and reports both energy errors, the
    position deviation and the split agreement of the final state."""
    import numpy as np
    import hhs
    steps = int(round(a.t_end / a.dt))
    ics = hhs.plummer(a.n, a.seed, getattr(a, "mass", 0))
    e0 = hhs.energy_host(ics)
    out = {}
    res = {}
    for name, prec in (("mixed", hhs.PREC_MIXED), ("fp64", hhs.PREC_FP64)):
        ctx = hhs.Context(a.n, 64, eta=a.eta)
        if tuning:
            ctx.set_tuning(**{k: v for k, v in tuning.items() if k != "ms_per_step"})
        d = hhs.ParticleSystem(a.n)
        d.upload(ics)
        ev = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
        torch.cuda.synchronize()
        ev[0].record()
        for _ in range(steps):
            hhs.hold_step(ctx, d, a.n, 0.0, a.dt, True, prec)
        ev[1].record()
        ctx.check()
        res[name] = d.download()
        e1 = hhs.energy_host(res[name])
        st = ctx.stats()
        out[name] = {"dE_over_E": (e1 - e0) / e0, "seconds": ev[0].elapsed_time(ev[1]) * 1e-3,
                     "steps_per_s": steps / (ev[0].elapsed_time(ev[1]) * 1e-3),
                     "nodes_per_step": st["nodes"] / steps, "max_level": st["max_level"],
                     "simtime": ctx.simtime()}
    m, f = res["mixed"], res["fp64"]
    dx = max(float(np.max(np.abs(m[k] - f[k]))) for k in ("x", "y", "z"))
    rel_ts = np.abs(m["ts"] - f["ts"]) / f["ts"]
    return {"metric": "accuracy of the mixed-precision HOLD against FP64 after t_end",
            "value": abs(out["mixed"]["dE_over_E"]), "unit": "|dE/E| (mixed)",
            "n": a.n, "eta": a.eta, "dt_top": a.dt, "t_end": a.t_end, "steps": steps,
            "results": out, "max_abs_dx_mixed_vs_fp64": dx,
            "median_rel_ts_diff": float(np.median(rel_ts)),
            "speedup_mixed_vs_fp64_device": out["mixed"]["steps_per_s"] / out["fp64"]["steps_per_s"]}


def run_side_measurements(a, torch, res):
    """Short measurements beside the headline, each well under a minute of GPU time:
    - config 2's acceptance numbers: the same sphere integrated to t = 1 (64 top-level
      steps) in mixed precision and on the FP64 device schedule (bit-exact with the CPU
      oracle), |dE/E| of both and max |dx| between the final states;
    - the scan of 2^28 Bernoulli(0.5) int32 flags (8 B per element) and stream
      compaction, checked bit for bit against the reference's own scan on the same GPU;
    - config 1 (N=1024 FP64 to t=1, bit for bit against the CPU oracle), config 3
      (N=65536 Salpeter) and config 5 (N=262144 90/10 masses) step rates;
    - config 3 through the multi-GPU step (hhs.DistHold) on a one-rank NCCL group;
    - the batched workload (512 clusters, N log-uniform in [64, 4096]): cluster steps/s,
      and the per-cluster energy errors at t=0.5 in mixed precision and FP64."""
    out = {}
    v = run_validate(argparse.Namespace(**{**vars(a), "t_end": 1.0}), torch, res.get("tuning"))
    out["accuracy_t1"] = {
        "t_end": 1.0, "steps": v["steps"],
        "dE_over_E_t1": v["results"]["mixed"]["dE_over_E"],
        "dE_over_E_t1_fp64": v["results"]["fp64"]["dE_over_E"],
        "max_dx_vs_fp64": v["max_abs_dx_mixed_vs_fp64"],
        "median_rel_ts_diff_vs_fp64": v["median_rel_ts_diff"],
        "target": "|dE/E| <= 1e-6 after one N-body time"}
    out["dE_over_E_t1"] = out["accuracy_t1"]["dE_over_E_t1"]
    out["max_dx_vs_fp64"] = out["accuracy_t1"]["max_dx_vs_fp64"]
    sc = run_scan(argparse.Namespace(**{**vars(a), "scan_log2n": 28, "steps": 5}), torch)
    row = sc["sweep"][0]
    hbm, src = hbm_peak()
    out["scan_2p28"] = {"n": 1 << 28, "p": 0.5, "scan_GBps": row["scan_GBps"],
                        "scan_frac_of_hbm": row["scan_GBps"] / hbm,
                        "compact_GBps": row["compact_GBps"],
                        "hbm_peak_GBps": hbm, "hbm_peak_source": src,
                        "bytes_per_element": 8,
                        "scan_properties_ok": row["scan_properties_ok"],
                        "bit_exact_vs_reference": row.get("bit_exact_vs_reference"),
                        "reference_scan_GBps": row.get("reference_scan_GBps")}
    torch.cuda.empty_cache()
    p1 = run_plain1k(a, torch)
    out["plain1k"] = {k: p1[k] for k in ("value", "unit", "steps", "gpu_steps_per_s",
                                         "cpu_oracle_steps_per_s", "cpu_threads",
                                         "bit_exact_gpu_vs_oracle", "dE_over_E")}
    out["plain1k"]["workload"] = "Plummer N=1024 FP64, eta=0.03, to t=1 (config 1)"
    out["deep_65536"] = time_engine(torch, 65536, 0.02, 1, a.dt, 3, 1)
    out["deep_65536"]["workload"] = ("Plummer N=65536 Salpeter masses, eta=0.02, mixed "
                                     "(config 3)")
    dist = time_dist(torch, 65536, 0.02, 1, a.dt, 3, 1)
    if dist is not None:
        dist["vs_device_step"] = dist["s_per_step"] / out["deep_65536"]["s_per_step"]
        dist["workload"] = ("config 3 through hhs.DistHold on a one-rank NCCL group, against "
                            "deep_65536 (the device-resident step)")
        out["dist_65536"] = dist
    out["large_262144"] = time_engine(torch, 262144, 0.02, 2, a.dt, 2, 1)
    out["large_262144"]["workload"] = ("Plummer N=262144 90/10 masses, eta=0.02, mixed "
                                       "(config 5)")
    out["batched_accuracy_t05"] = run_batched_accuracy(a, torch)
    b = run_batched(argparse.Namespace(**{**vars(a), "steps": 5, "warmup": 3}), torch)
    out["batched_512"] = {k: b[k] for k in ("value", "unit", "ms_per_step", "steps",
                                            "pair_interactions_per_s", "dE_over_E_after_steps")}
    out["batched_512"]["n_total"] = b["config"]["n_total"]
    out["batched_512"]["autotuned"] = b["config"]["autotuned"]
    out["batched_512"]["tuning"] = (b["config"]["autotune"] or {}).get("chosen")
    return out


def time_engine(torch, n, eta, mass, dt, steps, warmup, seed=2024):
    """Mixed-precision device steps of one seeded sphere (default tuning): steps/s, pair
    interactions/s and the hierarchy, timed with CUDA events on the launching stream."""
    import hhs
    s = hhs.plummer(n, seed, mass)
    ctx = hhs.Context(n, 64, eta=eta)
    d = hhs.ParticleSystem(n)
    stream = torch.cuda.Stream()
    sh = ctypes.c_void_p(stream.cuda_stream)
    d.upload(s, stream=sh)
    with torch.cuda.stream(stream):
        for _ in range(warmup):
            hhs.hold_step(ctx, d, n, 0.0, dt, True, hhs.PREC_MIXED, stream=sh)
        ctx.check(sh)
        ctx.reset_stats(sh)
        ev = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
        torch.cuda.synchronize()
        ev[0].record(stream)
        for _ in range(steps):
            hhs.hold_step(ctx, d, n, 0.0, dt, True, hhs.PREC_MIXED, stream=sh)
        ev[1].record(stream)
        torch.cuda.synchronize()
        ctx.check(sh)
    sec = ev[0].elapsed_time(ev[1]) * 1e-3
    st = ctx.stats(sh)
    ctx.destroy()
    d.free()
    return {"steps_per_s": steps / sec, "s_per_step": sec / steps, "steps": steps,
            "warmup": warmup, "pair_interactions_per_s": (st["kick_pairs"] + st["ts_pairs"]) / sec,
            "kick_pairs_per_step": st["kick_pairs"] / steps, "nodes_per_step": st["nodes"] / steps,
            "max_level": st["max_level"]}


def time_dist(torch, n, eta, mass, dt, steps, warmup, seed=2024):
    """The multi-GPU step (hhs.DistHold: timestep and kick launches split by sink, every
    result stored into each replica by the kernels, host barriers between launches) on a
    one-rank NCCL group, timed with CUDA events on the library's stream like the device
    step. With one rank every launch is a whole level, so the gap to the device step is the
    cost of the host-driven schedule and its barriers."""
    import datetime
    import socket
    import torch.distributed as tdist
    import hhs
    if tdist.is_available() and tdist.is_initialized():
        return None
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    tdist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0,
                             world_size=1, timeout=datetime.timedelta(seconds=120))
    try:
        s = hhs.plummer(n, seed, mass)
        ctx = hhs.Context(n, 64, eta=eta)
        d = hhs.ParticleSystem(n)
        d.upload(s)
        dh = hhs.DistHold(ctx, d)
        st = torch.cuda.default_stream()
        for _ in range(warmup):
            dh.step(n, dt, True, hhs.PREC_MIXED)
        torch.cuda.synchronize()
        ctx.check()
        ev = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
        ev[0].record(st)
        for _ in range(steps):
            dh.step(n, dt, True, hhs.PREC_MIXED)
        ev[1].record(st)
        torch.cuda.synchronize()
        ctx.check()
        sec = ev[0].elapsed_time(ev[1]) * 1e-3
        dh.close()
        ctx.destroy()
        d.free()
    finally:
        tdist.destroy_process_group()
    return {"s_per_step": sec / steps, "steps": steps, "warmup": warmup, "ranks": 1,
            "backend": "nccl", "min_pairs": 1 << 24}


def run_batched_accuracy(a, torch, t_end=0.5):
    """The batched workload integrated to t_end in mixed precision and in FP64 from the same
    initial conditions: the per-cluster |dE/E| of both, and of their difference."""
    import numpy as np
    import hhs
    sizes = cluster_sizes(a.seed)
    parts = [hhs.plummer(int(sizes[k]), a.seed * 1000 + int(k)) for k in range(len(sizes))]
    e0 = np.array([hhs.energy_host(p) for p in parts])
    packed = {f: np.concatenate([p[f] for p in parts]) for f in hhs.FIELDS}
    n = int(sizes.sum())
    packed["id"] = np.arange(n, dtype=np.int32)
    off = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int32)
    steps = int(round(t_end / a.dt))
    de = {}
    for name, prec in (("mixed", hhs.PREC_MIXED), ("fp64", hhs.PREC_FP64)):
        d = hhs.ParticleSystem(n)
        d.upload(packed)
        b = hhs.Batch(off, 64, eta=a.eta)
        for _ in range(steps):
            b.step(d, a.dt, True, prec)
        b.check()
        out = d.download()
        e1 = np.array([hhs.energy_host({f: np.ascontiguousarray(out[f][off[k]:off[k + 1]])
                                        for f in ("x", "y", "z", "vx", "vy", "vz", "m")})
                       for k in range(len(sizes))])
        de[name] = (e1 - e0) / e0
        d.free()
    diff = np.abs(de["mixed"] - de["fp64"])
    q = lambda v: {"median": float(np.median(v)), "p90": float(np.percentile(v, 90)),
                   "max": float(np.max(v))}
    return {"t_end": t_end, "steps": steps, "clusters": len(sizes), "n_total": n,
            "abs_dE_over_E_mixed": q(np.abs(de["mixed"])), "abs_dE_over_E_fp64": q(np.abs(de["fp64"])),
            "abs_dE_over_E_mixed_minus_fp64": q(diff)}


def hbm_peak():
    """Measured HBM copy bandwidth of this pool's B200s (GB/s), else the fallback."""
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(peaks["hbm_gbs"]), "measured"
    except (OSError, ValueError, KeyError, TypeError):
        return 6650.0, "fallback"


def main():
    a = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if a.impl == "reference":
        out = run_reference(a, rank, world)
        if out is not None:
            print(json.dumps(out), flush=True)
        return
    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as d
        d.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                             device_id=torch.device("cuda", local))
        dist = d
    if a.workload == "large":
        a.n, a.eta, a.mass = 262144, 0.02, 2
    elif a.workload == "deep":
        a.n, a.eta, a.mass = 65536, 0.02, 1
    if a.workload == "batched":
        out = run_batched(a, torch, rank, world, dist)
        if rank == 0:
            print(json.dumps(out), flush=True)
        if dist is not None:
            dist.destroy_process_group()
        return
    if a.workload in ("scan", "validate", "plain1k", "kickprobe", "tsprobe"):
        if rank == 0:
            fn = {"scan": run_scan, "validate": run_validate, "plain1k": run_plain1k,
                  "kickprobe": run_kickprobe, "tsprobe": run_tsprobe}[a.workload]
            out = fn(a, torch)
            if a.workload == "scan" and "roofline" in out:
                hbm, src = hbm_peak()
                out["roofline"]["peak"] = hbm
                out["roofline"]["peak_source"] = src
                out["roofline"]["frac"] = out["value"] / hbm
            print(json.dumps(out), flush=True)
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
        return
    res = run_ours(a, rank, world, torch, dist)
    cpu = None
    extra = {}
    if rank == 0 and world == 1 and not a.no_baselines:
        ref = run_reference(argparse.Namespace(**{**vars(a), "steps": 1}), 0, 1, isolated=False)
        cpu = ref["cpu_baseline"]
        if a.workload == "plummer16k":
            extra = run_side_measurements(a, torch, res)
    if rank == 0:
        step_ms = res["t_ms"] / a.steps
        line = {
            "metric": METRIC, "value": res["value"], "unit": "HOLD steps/s", "n_gpus": world,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": step_ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32-pair/f64-state" if a.prec == "mixed" else "f64",
            "data": "synthetic (seeded Plummer sphere; no dataset)",
            "config": {"workload": workload_name(a), "n": a.n, "eta": a.eta, "dt_top": a.dt,
                       "precision": a.prec, "schedule": a.schedule,
                       "tuning": res["tuning"], "autotuned": res["autotune"] is not None,
                       "autotune": res["autotune"],
                       "l2": "flushed between timed steps (256 MiB memset)",
                       "parallelism": f"replicas x{world}"},
            "pair_interactions_per_s": res["pairs_per_step"] * res["value"],
            "pairs_per_step": res["pairs_per_step"],
            "hierarchy": {"nodes_per_step": res["stats"]["nodes"] / a.steps,
                          "max_level": res["stats"]["max_level"]},
            "dE_over_E_bench_run": res["dE_over_E"],
            "e2e": res["e2e"],
            "gpu_launches": res["launches"],
            "clocks": res["clocks"],
            "roofline": roofline(res, a, res["fma_peaks"], nominal_fp32_tflops(torch)),
            "kernel_profile": res["prof"],
            "fma_peaks_tflops": {"fp32": res["fma_peaks"][0], "fp64": res["fma_peaks"][1],
                                 "fp32x2_packed": res["fma2_peak"]},
            "cpu_baseline": cpu,
        }
        if "fp64_plain_steps_per_s" in res:
            line["fp64_plain_gpu"] = {"value": res["fp64_plain_steps_per_s"],
                                      "unit": "HOLD steps/s", "steps": res["fp64_plain_steps"],
                                      "schedule": "host-driven, one-thread-per-sink FP64"}
            line["speedup_vs_fp64_plain"] = res["value"] / res["fp64_plain_steps_per_s"]
        if "fp64_engine_steps_per_s" in res:
            line["fp64_device_schedule"] = {"value": res["fp64_engine_steps_per_s"],
                                            "unit": "HOLD steps/s"}
            line["speedup_vs_fp64_device_schedule"] = res["value"] / res["fp64_engine_steps_per_s"]
        line.update(extra)
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
