#!/usr/bin/env python
"""Benchmark of the SPME RPY mobility + block-Lanczos Brownian-dynamics hot path.

Metric (headline): Brownian-dynamics steps per second at N = 100,000
(volume fraction 0.2, 256^3 grid, p = 6), M.f within 1e-6 and sqrt(M) z within
1e-5 of FP64.  One bench "step" is one mobility interval of the reference's
BD integrator (BDSimBox::Advance, src/simbox/simbox_bd.cc:296-366 of the
reference) with mob-interval 16:
    Update(pos) ; Y = sqrt(M) Z (block Lanczos, 16 RHS, tol 1e-6) ;
    16 x { disp_s = dt M F_s + sqrt(2 dt) Y_s ; pos += disp_s }
i.e. 16 BD steps.  F and Z are i.i.d. N(0,1), resident in HBM for `value`;
`e2e` runs the same interval through the host-pointer C ABI with pinned host
buffers (H2D of pos, Z, F, Y in / D2H of Y, disp every step).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

For N > 1 (launched by torchrun) every rank runs an independent replica
system (weak scaling, no data-path collective); the timed region is bracketed
by barriers and the reported time is the max over ranks.

At N = 1 the config-2 line also carries `other_configs`: short runs of
config 3 (trajectory), config 4 (batched systems) and config 5 (served
stream), each a child process started after the config-2 measurement with
its own timing and clock record (--no-other-configs skips them; each also
runs alone with --workload cfg3|cfg4|cfg5).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "BD steps/s & M·f products/s at N=1e5, rel err ≤1e-6 vs FP64; p50/p99 latency"
UNIT = "BD steps/s"
INTERVAL = 16          # mob-interval: BD steps per bench step (= Lanczos RHS)
DT = 1e-3              # BD time step (a = kT = 6 pi eta = 1 units)
PEAKS_FALLBACK = {"hbm_gbs": 6650.0}


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--workload", default="cfg2",
                    help="cfg2 (default), cfg3 (trajectory), cfg4 (batch), cfg5 (served stream)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-full-interval", action="store_true",
                    help="reference arm: skip the one whole measured interval (samples only)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-compare", action="store_true",
                    help="config 4: skip the lanes-mode and plain per-system comparison legs")
    ap.add_argument("--profile-case", action="store_true",
                    help="small case for ncu: a few mobility products, no timing output")
    ap.add_argument("--profile-rhs", type=int, default=1, help="RHS per product in --profile-case")
    ap.add_argument("--no-other-configs", action="store_true",
                    help="config 2 at N=1: skip the short config 3/4/5 legs attached to the line")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# clocks
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(prefix="clocks_", suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as fh:
            for line in fh:
                t = [x.strip() for x in line.split(",")]
                if len(t) < 9:
                    continue
                try:
                    sm.append(float(t[1]))
                    smax = float(t[2])
                except ValueError:
                    continue
                for name, val in zip(names, t[5:9]):
                    if val.lower().startswith("active"):
                        reasons.add(name)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        return d, "measured"
    return PEAKS_FALLBACK, "fallback"


# ---------------------------------------------------------------------------
# algorithmic bytes per stage (one launch covering `nr` RHS)
# ---------------------------------------------------------------------------
# kernel behind each profiled stage of a 16-RHS product (K = 256: the
# tensor-core spread takes calls of >= 8 RHS)
STAGE_KERNEL = {"gather_forces": "k_gather_both", "real_space": "k_pair_apply<16>",
                "spread_tc": "k_spread_tc<K,16>", "spread_xfwd": "k_spread_xfwd<K>",
                "yfft_fwd": "k_ypass_tma<K,fwd>", "zfft_influence": "k_zpass_fused_tma<K>",
                "yfft_inv": "k_ypass_tma<K,inv>", "xinv_interp": "k_xinv_interp<K>", "combine": "k_combine"}


def rename_stages(stages: dict, K: int, nr: int) -> dict:
    """The library's stage 'spread_x' is the tensor-core spread for K = 256
    and >= 8 RHS, the shared-memory spread + x FFT otherwise."""
    tc = K == 256 and nr >= 8 and os.environ.get("STOKESDT_NO_TC", "0") != "1"
    return {("spread_tc" if tc else "spread_xfwd") if k == "spread_x" else k: v for k, v in stages.items()}


def cufft_reference_ms(K: int, ngrids: int, dev, reps: int = 3):
    """cuFFT (torch.fft) r2c and c2r of `ngrids` K^3 FP32 grids on the
    current stream: the library FFT the hand-written passes stand beside
    (timing reference only; cuFFT is not on the product path)."""
    import torch
    x = torch.randn((ngrids, K, K, K), dtype=torch.float32, device=dev)
    out = {}
    X = torch.fft.rfftn(x, dim=(1, 2, 3))          # warm-up (plan creation)
    torch.fft.irfftn(X, s=(K, K, K), dim=(1, 2, 3))
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    torch.cuda.synchronize(dev)
    ev[0].record()
    for _ in range(reps):
        X = torch.fft.rfftn(x, dim=(1, 2, 3))
    ev[1].record()
    for _ in range(reps):
        y = torch.fft.irfftn(X, s=(K, K, K), dim=(1, 2, 3))
    ev[2].record()
    torch.cuda.synchronize(dev)
    out["r2c_ms"] = round(ev[0].elapsed_time(ev[1]) / reps, 4)
    out["c2r_ms"] = round(ev[1].elapsed_time(ev[2]) / reps, 4)
    del x, X, y
    torch.cuda.empty_cache()
    return out


def stage_bytes(stage: str, N: int, K: int, p: int, nr: int, pairs: int = 0) -> float:
    """Bytes a stage must move at minimum, per launch of nr RHS.  Ghat1 is one
    component's complex half-spectrum K*K*(K/2+1)*8 B; the real-space grid
    never reaches HBM (spreading feeds the x-FFT in shared memory and the
    inverse x-FFT feeds the interpolation).  With a stored real-space pair
    list (`pairs` > 0) the real-space stage streams 24 B per pair, reads the
    float4 force rows once and writes the FP32 result."""
    g1 = K * K * (K // 2 + 1) * 8.0
    part = N * (4 + 3 * p * 4.0)            # packed base index + spline weights
    if stage in ("spread_xfwd", "spread_tc"):
        return 3 * nr * g1 + part + 3 * nr * N * 4.0
    if stage in ("yfft_fwd", "yfft_inv"):
        return 2 * 3 * nr * g1
    if stage == "zfft_influence":
        return 2 * 3 * nr * g1 + K * K * (K // 2 + 1) * 4.0
    if stage == "xinv_interp":
        return 3 * nr * g1 + part + 3 * nr * N * 4.0
    if stage == "real_space":
        if pairs > 0:
            return 24.0 * pairs + N * (8.0 + 4.0 + 16.0 * nr) + 12.0 * nr * N
        return N * (32.0 + 12.0 * nr) + 12.0 * nr * N
    if stage == "gather_forces":
        return 3 * nr * N * (8.0 + 8.0)
    if stage == "combine":
        return 3 * nr * N * (8.0 + 4 + 4 + 8 + 8)
    return 0.0


# ---------------------------------------------------------------------------
# CPU baseline: the reference's own code (oracle/_ref) on a bounded sample
# ---------------------------------------------------------------------------
def cpu_sample(w, pos, its_hint):
    """Times Update + one 2-RHS MulVector of the reference (or the numpy port
    when the reference library is absent) on all host cores and extrapolates
    one mobility interval: T_update + (iters + 1) * 16 * T_mulvec(1 RHS)."""
    from oracle import ref
    N = w.npos
    rdi = np.ones(N)
    n3 = 3 * N
    f = np.random.default_rng(w.seed_f).standard_normal((2, n3))
    if ref.available():
        kind = "reference"
        mob = ref.RefMob.spme(rdi, w.box, w.xi, w.rmax, w.dim, w.porder)
        t0 = time.perf_counter()
        mob.update(pos, rdi)
        t1 = time.perf_counter()
        mob.mulvec(f)
        t2 = time.perf_counter()
        mob.close()
    else:
        from oracle import spme_oracle as so
        kind = "port"
        o = so.SpmeOracle(rdi, w.box, w.xi, w.rmax, w.dim, w.porder)
        t0 = time.perf_counter()
        o.update(pos)
        t1 = time.perf_counter()
        o.mulvec(f)
        t2 = time.perf_counter()
    t_up, t_mv1 = t1 - t0, (t2 - t1) / 2.0
    iters = its_hint
    t_interval = t_up + (iters + 1) * INTERVAL * t_mv1 + INTERVAL * t_mv1
    return {
        "value": INTERVAL / t_interval, "unit": UNIT, "cores": os.cpu_count(), "kind": kind,
        "sample": (f"Update + one 2-RHS MulVector at N={N} ({t_up:.2f} s + {2 * t_mv1:.2f} s on "
                   f"{os.cpu_count()} threads), extrapolated to one mobility interval = Update + "
                   f"{iters + 1} block-Lanczos iterations x {INTERVAL} RHS + {INTERVAL} M.F products "
                   f"(Lanczos host work and reorthogonalisation not charged to the reference)"),
        "t_update_s": t_up, "t_mulvec_per_rhs_s": t_mv1, "lanczos_iters_assumed": iters,
    }


# the reference's own block Lanczos iteration count for cfg2 (BrwnLanczos,
# 16 RHS, tol 1e-6, maxiters 100), measured once by running oracle/_ref to
# convergence on the same inputs; used by the reference arm's extrapolation.
REF_ITERS = {"cfg2": 75}


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as fh:
            for line in fh:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def reference_full_interval(w, pos):
    """One whole mobility interval through the reference's own code on all
    host cores (BDSimBox::Advance, src/simbox/simbox_bd.cc:307-339):
    MobSpme::Update, BrwnLanczos::Compute on 16 N(0,1) vectors (tol, 100
    iterations at most), then 16 x { MulVector(1, dt, F_s, sqrt(2 dt), Y_s) ;
    pos += Y_s }.  The reference's block Lanczos keeps ~21 MB on the stack
    (src/brwn/brwn_lanczos.cc:97), so it runs on a thread with a 256 MB
    stack.  Returns the wall time, the shim FFT's share and the iteration
    count the reference logged."""
    import threading
    from oracle import ref
    N, n3 = w.npos, 3 * w.npos
    rdi = np.ones(N)
    Z = np.random.default_rng(w.seed_z).standard_normal((INTERVAL, n3))
    F = np.random.default_rng(w.seed_f).standard_normal((INTERVAL, n3))
    out = {}

    def run():
        mob = ref.RefMob.spme(rdi, w.box, w.xi, w.rmax, w.dim, w.porder)
        lz = ref.RefLanczos(n3, w.max_iters, INTERVAL, w.lanczos_tol)
        p = np.ascontiguousarray(pos.reshape(-1), dtype=np.float64).copy()
        ref.shim_fft_seconds(reset=True)
        t0 = time.perf_counter()
        mob.update(np.mod(p, w.box), rdi)
        t1 = time.perf_counter()
        Y, its = lz.compute(mob, Z)
        t2 = time.perf_counter()
        sq = math.sqrt(2.0 * DT)
        for k in range(INTERVAL):
            disp = mob.mulvec(F[k], DT, sq, Y[k])[0]
            p += disp
        t3 = time.perf_counter()
        fft_s, calls = ref.shim_fft_seconds()
        out.update(total_s=t3 - t0, update_s=t1 - t0, lanczos_s=t2 - t1, steps_s=t3 - t2, fft_s=fft_s,
                   fft_calls=calls, iters=its)
        mob.close()
        lz.close()

    threading.stack_size(256 << 20)
    th = threading.Thread(target=run)
    th.start()
    th.join()
    threading.stack_size(0)
    return out


def mkl_fft_pair_s(K: int) -> float:
    """Seconds of one FP64 K^3 forward r2c plus backward c2r with torch's CPU
    FFT (MKL-backed in this build) on all host threads: an MKL-class figure
    for the transforms the reference runs through MKL DFTI."""
    import torch
    torch.set_num_threads(os.cpu_count() or 1)
    x = torch.randn((K, K, K), dtype=torch.float64)
    X = torch.fft.rfftn(x)
    torch.fft.irfftn(X, s=(K, K, K))
    reps = 3
    t0 = time.perf_counter()
    for _ in range(reps):
        X = torch.fft.rfftn(x)
        torch.fft.irfftn(X, s=(K, K, K))
    return (time.perf_counter() - t0) / reps


def run_reference(args):
    """The reference arm: the reference's own CPU path (oracle/_ref, built
    from its unmodified sources) on this box's host cores.  Every timed step
    is a bounded sample (Update + one 2-RHS MulVector) that gives the
    extrapolated interval; after the timed steps one whole interval runs
    through the reference's own Update, BrwnLanczos::Compute and MulVector,
    and `value` is that measured interval (16 BD steps / its wall time)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from stokesdt_b200 import workloads as wl
    w = wl.WORKLOADS[args.workload]
    pos = wl.rsa_positions(w.npos, w.box, w.seed_pos)
    its = REF_ITERS.get(args.workload) or 20
    samples = []
    t_steps = 0.0
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        s = cpu_sample(w, pos, its)
        if i >= args.warmup:
            samples.append(s)
            t_steps += time.perf_counter() - t0
    v_extrap = float(np.median([s["value"] for s in samples]))
    base = dict(samples[-1])
    cpu = {"value": v_extrap, "unit": UNIT, "cores": os.cpu_count(), "kind": base["kind"],
           "sample": base["sample"], "cpu_model": cpu_model(),
           "extrapolated_interval_s": round(INTERVAL / v_extrap, 3)}
    value = v_extrap
    if not args.no_full_interval and base["kind"] == "reference":
        full = reference_full_interval(w, pos)
        value = INTERVAL / full["total_s"]
        mkl_pair = mkl_fft_pair_s(w.dim)
        mkl_equiv = 0.5 * full["fft_calls"] * mkl_pair
        adjusted = full["total_s"] - full["fft_s"] + mkl_equiv
        cpu.update({
            "value": value,
            "measured_interval_s": round(full["total_s"], 3),
            "measured_split_s": {"update": round(full["update_s"], 3), "lanczos": round(full["lanczos_s"], 3),
                                 "16_steps": round(full["steps_s"], 3)},
            "reference_lanczos_iters": full["iters"],
            "measured_over_extrapolated": round(full["total_s"] / (INTERVAL / v_extrap), 4),
            "fft_share": round(full["fft_s"] / full["total_s"], 4),
            "fft_s": round(full["fft_s"], 3), "fft_calls": full["fft_calls"],
            "mkl_class_fft_pair_s": round(mkl_pair, 4),
            "fft_adjusted_interval_s": round(adjusted, 3),
            "value_fft_adjusted": INTERVAL / adjusted,
            "sample": (f"timed steps: {base['sample']}; value: one whole mobility interval measured through "
                       f"the reference's own MobSpme::Update, BrwnLanczos::Compute (16 RHS, tol "
                       f"{w.lanczos_tol}) and 16 MulVector calls on {os.cpu_count()} threads"),
        })
        log(f"reference interval: {full['total_s']:.1f} s measured vs {INTERVAL / v_extrap:.1f} s "
            f"extrapolated; shim FFT {full['fft_s']:.1f} s of it")
    out = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * t_steps / max(1, args.steps), 3),
        "ms_per_interval": round(1e3 * INTERVAL / value, 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": workload_config(w),
        "cpu_baseline": cpu,
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out))


def workload_config(w):
    return {"workload": w.name, "npos": w.npos, "phi": w.phi, "box": round(w.box, 6), "K": w.dim,
            "porder": w.porder, "xi": w.xi, "rmax": round(w.rmax, 6), "nrhs": w.nrhs,
            "lanczos_tol": w.lanczos_tol, "lanczos_max_iters": w.max_iters,
            "lanczos_reorth": w.reorth, "dt": DT,
            "step": "one mobility interval = Update + 16-RHS block Lanczos + 16 x (M.F + pos update)",
            "l2": "no flush: the 16-RHS grids (3.3 GB) exceed the 126 MB L2",
            "parallelism": "replicas (one independent system per GPU)"}


# ---------------------------------------------------------------------------
# B200 arm
# ---------------------------------------------------------------------------
def log(msg):
    print(f"[bench] {msg}", file=sys.stderr, flush=True)


# ---------------------------------------------------------------------------
# multi-rank helpers (replicas: one independent system per rank, no exchange)
# ---------------------------------------------------------------------------
def replica_seed(base: int, rank: int) -> int:
    """Seed of rank's independent replica system."""
    return base + 1000 * rank


def max_over_ranks(dist, x: float, device) -> float:
    """The slowest rank's time: the whole job finishes when it does."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(world: int, units_per_rank: float, max_ms: float) -> float:
    """Whole-job throughput: units processed by all ranks / slowest rank's time."""
    return world * units_per_rank / (max_ms / 1e3)


def run_b200(args):
    import torch
    import stokesdt_b200 as sdt
    from stokesdt_b200 import workloads as wl

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))

    w = wl.WORKLOADS[args.workload]
    N, L, K, p = w.npos, w.box, w.dim, w.porder
    n3 = 3 * N
    pos0 = wl.rsa_positions(N, L, replica_seed(w.seed_pos, rank))
    Z = np.random.default_rng(replica_seed(w.seed_z, rank)).standard_normal((INTERVAL, n3))
    F = np.random.default_rng(replica_seed(w.seed_f, rank)).standard_normal((INTERVAL, n3))

    dev = torch.device("cuda", local)
    # a dedicated stream: the legacy default stream's handle is 0, which the C
    # ABI reads as "use the engine's own stream"
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    mob = sdt.MobSpme(N, np.ones(N), L, w.xi, w.rmax, K, p, device=local)
    if not mob.Init():
        raise RuntimeError(f"MobSpme Init failed: {mob.last_error}")
    mob.set_stream(stream.cuda_stream)

    d_pos = torch.tensor(pos0.ravel(), device=dev)
    d_Z = torch.tensor(Z, device=dev)
    d_F = torch.tensor(F, device=dev)
    d_Y = torch.empty((INTERVAL, n3), dtype=torch.float64, device=dev)
    if args.profile_case:
        # two products only (for profiler captures): no Lanczos workspace
        mob.update_device(d_pos.data_ptr())
        for _ in range(2):
            mob.mulvec_device(0, args.profile_rhs, 1.0, n3, d_Z.data_ptr(), 0.0, n3, d_Y.data_ptr())
        torch.cuda.synchronize(dev)
        return
    lz = sdt.BrwnLanczos(n3, w.max_iters, INTERVAL, w.lanczos_tol, device=local, reorth=w.reorth)
    if not lz.Init():
        raise RuntimeError("BrwnLanczos Init failed")
    lz.set_stream(stream.cuda_stream)
    sq = math.sqrt(2.0 * DT)
    iters_seen = []

    d_pos0 = d_pos.clone()

    def interval():
        # every bench step starts from the same configuration so the workload
        # (and the Lanczos iteration count) stays fixed; positions are then
        # advanced within the step as BDSimBox::Advance does
        d_pos.copy_(d_pos0)
        mob.update_device(d_pos.data_ptr())
        its = lz.compute_device(mob, INTERVAL, n3, d_Z.data_ptr(), n3, d_Y.data_ptr())
        iters_seen.append(its[0])
        for s in range(INTERVAL):
            mob.mulvec_device(0, 1, DT, n3, d_F[s].data_ptr(), sq, n3, d_Y[s].data_ptr())
            d_pos.add_(d_Y[s])

    def barrier():
        torch.cuda.synchronize(dev)
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(dev)

    def max_ranks(x: float) -> float:
        return max_over_ranks(dist, x, dev)

    log(f"rank {rank}: N={N} K={K} setup done, warm-up")
    for _ in range(args.warmup):
        interval()
    barrier()
    sampler = ClockSampler(local)
    sampler.start()
    launches0 = sdt.kernel_launches()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    barrier()
    ev[0].record(stream)
    for k in range(args.steps):
        interval()
        ev[k + 1].record(stream)
    torch.cuda.synchronize(dev)
    barrier()
    clocks = sampler.stop()
    launches = sdt.kernel_launches() - launches0
    step_ms = [ev[k].elapsed_time(ev[k + 1]) for k in range(args.steps)]
    total_ms = max_ranks(ev[0].elapsed_time(ev[-1]))
    value = aggregate_rate(world, INTERVAL * args.steps, total_ms)
    log(f"timed {args.steps} intervals: {total_ms:.1f} ms, iters {iters_seen[-args.steps:]}")

    # M.f products per second: 16-RHS products back to back, device resident
    mob.update_device(d_pos.data_ptr())
    reps = 5
    mob.mulvec_device(0, INTERVAL, 1.0, n3, d_Z.data_ptr(), 0.0, n3, d_Y.data_ptr())
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        mob.mulvec_device(0, INTERVAL, 1.0, n3, d_Z.data_ptr(), 0.0, n3, d_Y.data_ptr())
    e1.record(stream)
    torch.cuda.synchronize(dev)
    mf_ms = max_ranks(e0.elapsed_time(e1))
    mf_per_s = aggregate_rate(world, INTERVAL * reps, mf_ms)

    # per-stage profile and roofline of the dominant kernel
    log(f"M.f 16 RHS: {mf_ms / reps:.3f} ms")
    stages = rename_stages(mob.profile(INTERVAL, 3), K, INTERVAL)
    log(f"stages: {stages}")
    dom = max((k for k in stages if k != "combine"), key=lambda k: stages[k])
    peaks, peak_kind = measured_peaks()
    pairs = max(0, mob.pairlist_size())
    algo = stage_bytes(dom, N, K, p, INTERVAL, pairs)
    achieved = algo / (stages[dom] / 1e3) / 1e9
    traffic = None
    tp = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tp):
        with open(tp) as fh:
            tj = json.load(fh)
        if dom in tj:
            traffic = tj[dom]["bytes_per_launch_at_bench_size"]
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peaks["hbm_gbs"],
                "unit": "GB/s", "frac": round(achieved / peaks["hbm_gbs"], 4), "traffic": traffic,
                "kernel": STAGE_KERNEL.get(dom, dom).replace("<K>", f"<{K}>"), "stage": dom,
                "peak_source": peak_kind,
                "algorithmic_bytes_per_launch": algo, "launch_ms": round(stages[dom], 4)}
    # the whole 16-RHS product against the unfused per-RHS figure 4G + 4Ghat + T
    # (real grid G = 3 K^3 4 B, half spectrum Ghat = 3 K^2 (K/2+1) 8 B, table
    # T = K^2 (K/2+1) 8 B): fused stage boundaries count as work done
    unfused = 4 * 3 * K ** 3 * 4 + 4 * 3 * K * K * (K // 2 + 1) * 8 + K * K * (K // 2 + 1) * 8
    mf_gbs = INTERVAL * unfused / (mf_ms / reps / 1e3) / 1e9
    roofline_mf = {"bound": "hbm", "achieved": round(mf_gbs, 1), "peak": peaks["hbm_gbs"], "unit": "GB/s",
                   "frac": round(mf_gbs / peaks["hbm_gbs"], 4), "peak_source": peak_kind,
                   "unfused_bytes_per_rhs": unfused, "product_ms": round(mf_ms / reps, 4)}

    # cuFFT beside the hand-written chain: r2c + c2r of the 3 x 16 grids of
    # one 16-RHS product (the chain's transforms are fused with the spread,
    # the influence multiply and the interpolation)
    cufft = None
    try:
        cufft = cufft_reference_ms(K, 3 * INTERVAL, dev)
        chain = ("spread_tc", "spread_xfwd", "yfft_fwd", "zfft_influence", "yfft_inv", "xinv_interp")
        cufft["ngrids"] = 3 * INTERVAL
        cufft["hand_written_chain_ms"] = round(sum(stages.get(k, 0.0) for k in chain), 4)
        cufft["note"] = ("hand_written_chain_ms includes the spread, the influence multiply and the "
                         "interpolation fused into the transforms; cuFFT's r2c + c2r are transforms only")
        log(f"cuFFT reference: {cufft}")
    except Exception as exc:  # noqa: BLE001 (timing reference only)
        log(f"cuFFT reference skipped: {exc}")

    # end to end through the host-pointer C ABI (pinned host buffers)
    e2e = None
    if not args.no_e2e:
        hp = torch.empty(n3, dtype=torch.float64).pin_memory().numpy()
        hp[:] = pos0.ravel()
        hZ = torch.tensor(Z).pin_memory().numpy()
        hF = torch.tensor(F).pin_memory().numpy()
        hY = torch.empty((INTERVAL, n3), dtype=torch.float64).pin_memory().numpy()

        hp0 = hp.copy()

        def interval_host():
            hp[:] = hp0
            mob.Update(hp)
            lz.Compute(mob, INTERVAL, n3, hZ, n3, hY)
            for s in range(INTERVAL):
                mob.MulVector(1, DT, n3, hF[s], sq, n3, hY[s])
                np.add(hp, hY[s], out=hp)

        interval_host()
        barrier()
        ke = max(1, min(args.steps, 3))
        h0, h1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        h0.record(stream)
        for _ in range(ke):
            interval_host()
        h1.record(stream)
        torch.cuda.synchronize(dev)
        barrier()
        e_ms = max_ranks(h0.elapsed_time(h1))
        h2d = 8 * n3 * (1 + INTERVAL + 2 * INTERVAL)
        d2h = 8 * n3 * (INTERVAL + INTERVAL)
        e2e = {"value": aggregate_rate(world, INTERVAL * ke, e_ms), "unit": UNIT,
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "steps": ke}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        its_hint = REF_ITERS.get(args.workload) or int(np.median(iters_seen))
        cpu = cpu_sample(w, pos0, its_hint)
        cpu = {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")}

    if rank == 0:
        lat = np.array(step_ms)
        out = {
            "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(total_ms / args.steps, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
            "data": "synthetic", "config": workload_config(w),
            "roofline": roofline, "roofline_mf": roofline_mf, "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": int(launches),
            "clocks": clocks,
            "mf_products_per_s": round(mf_per_s, 1),
            "latency_ms": {"p50": round(float(np.percentile(lat, 50)), 3),
                           "p99": round(float(np.percentile(lat, 99)), 3)},
            "lanczos_iters": iters_seen[-args.steps:],
            "stage_ms_16rhs": {k: round(v, 4) for k, v in stages.items()},
            "cufft_reference": cufft,
        }
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return out if rank == 0 else None


# short legs of configs 3-5 run after the config-2 line's own measurement (N=1
# only), each its own process with its own clock record: (workload, args, timeout s)
OTHER_CONFIGS = (("cfg3", ["--steps", "20", "--warmup", "3", "--no-cpu-baseline"], 600),
                 ("cfg4", ["--steps", "1", "--warmup", "3"], 900),
                 ("cfg5", ["--steps", "5", "--warmup", "3"], 600))
OTHER_KEYS = ("metric", "value", "unit", "ms_per_step", "higher_is_better", "e2e", "clocks", "gpu_launches",
              "latency_ms", "lanes_mode_systems_per_s_rank0", "plain_per_system_systems_per_s_rank0",
              "packed_over_plain", "phase_ms_rank0", "per_rate", "plain_per_request_path", "batching_rank0",
              "lanczos_iters_median", "roofline")


def run_other_configs():
    """Run the short config 3/4/5 legs as child processes and keep the main
    fields of their JSON lines (or the reason a leg gave none)."""
    import subprocess
    res = {}
    for wk, extra, tmo in OTHER_CONFIGS:
        cmd = [sys.executable, os.path.abspath(__file__), "--workload", wk, "--no-other-configs"] + extra
        t0 = time.perf_counter()
        try:
            p = subprocess.run(cmd, capture_output=True, text=True, timeout=tmo)
            line = [l for l in p.stdout.splitlines() if l.startswith("{")]
            if p.returncode != 0 or not line:
                res[wk] = {"error": f"exit {p.returncode}: {(p.stderr or '').strip()[-300:]}"}
            else:
                d = json.loads(line[-1])
                res[wk] = {k: d[k] for k in OTHER_KEYS if k in d}
                res[wk]["config"] = d.get("config", {}).get("workload")
        except subprocess.TimeoutExpired:
            res[wk] = {"error": f"did not finish within {tmo} s"}
        res[wk]["wall_s"] = round(time.perf_counter() - t0, 1)
        log(f"{wk}: {res[wk].get('value', res[wk].get('error'))}")
    return res


def run_b200_traj(args, w):
    """Config 3: a Brownian trajectory with steric repulsion through the
    device-resident integrator (sdt_bd_advance); one bench step = one BD step
    (Update + 1-RHS Lanczos + steric force + M.F + position update, as
    BDSimBox::Advance with mob-interval 1).  `e2e` keeps the positions on
    the host (pinned) and moves them in and out every step."""
    import torch
    import stokesdt_b200 as sdt
    from stokesdt_b200 import workloads as wl

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    N, n3 = w.npos, 3 * w.npos
    pos0 = wl.rsa_positions(N, w.box, replica_seed(w.seed_pos, rank)).reshape(-1)
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    mob = sdt.MobSpme(N, np.ones(N), w.box, w.xi, w.rmax, w.dim, w.porder, device=local)
    lz = sdt.BrwnLanczos(n3, w.max_iters, max(1, w.mob_interval), w.lanczos_tol, device=local,
                         reorth=w.reorth)
    st = sdt.StericForce(N, np.ones(N), w.box, w.steric_r0, w.steric_k0, device=local)
    if not (mob.Init() and lz.Init() and st.Init()):
        raise RuntimeError("engine Init failed")
    bd = sdt.BDIntegrator(mob, lz, st, dt=w.dt, mob_interval=w.mob_interval,
                          seed=replica_seed(w.seed_z, rank))
    bd.set_stream(stream.cuda_stream)
    bd.set_positions(pos0)

    def barrier():
        torch.cuda.synchronize(dev)
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(dev)

    bd.Advance(args.warmup)
    barrier()
    sampler = ClockSampler(local)
    sampler.start()
    launches0 = sdt.kernel_launches()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    ev[0].record(stream)
    for k in range(args.steps):
        bd.Advance(1)
        ev[k + 1].record(stream)
    torch.cuda.synchronize(dev)
    barrier()
    clocks = sampler.stop()
    launches = sdt.kernel_launches() - launches0
    step_ms = [ev[k].elapsed_time(ev[k + 1]) for k in range(args.steps)]
    total_ms = max_over_ranks(dist, ev[0].elapsed_time(ev[-1]), dev)
    value = aggregate_rate(world, args.steps, total_ms)
    info = bd.info()
    log(f"timed {args.steps} BD steps: {total_ms:.1f} ms, last Lanczos iterations {info['last_iters']}")

    e2e = None
    if not args.no_e2e:
        hp = torch.empty(n3, dtype=torch.float64).pin_memory().numpy()
        hp[:] = bd.get_positions()
        ke = max(1, min(args.steps, 5))
        barrier()
        h0, h1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        h0.record(stream)
        for _ in range(ke):
            bd.set_positions(hp)
            bd.Advance(1)
            hp[:] = bd.get_positions()
        h1.record(stream)
        torch.cuda.synchronize(dev)
        e_ms = max_over_ranks(dist, h0.elapsed_time(h1), dev)
        e2e = {"value": aggregate_rate(world, ke, e_ms), "unit": "BD steps/s",
               "h2d_bytes_per_step": 8 * n3, "d2h_bytes_per_step": 8 * n3, "steps": ke}

    if rank == 0:
        lat = np.array(step_ms)
        cfg = workload_config(w)
        cfg.update({"dt": w.dt, "steric_r0": w.steric_r0, "steric_k0": w.steric_k0,
                    "mob_interval": w.mob_interval,
                    "step": "one BD step = Update + 1-RHS Lanczos + steric force + M.F + pos update",
                    "l2": "no flush: per-step grids and pair list (~0.5 GB) exceed the 126 MB L2"})
        out = {
            "metric": "BD steps/s (config 3 trajectory)", "value": round(value, 3), "unit": "BD steps/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(total_ms / args.steps, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic", "config": cfg,
            "e2e": e2e, "gpu_launches": int(launches), "clocks": clocks,
            "latency_ms": {"p50": round(float(np.percentile(lat, 50)), 3),
                           "p99": round(float(np.percentile(lat, 99)), 3)},
            "lanczos_not_converged": info["not_converged"],
        }
        print(json.dumps(out))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def batch_units(systems, world: int, rank: int):
    """Config 4 sharding: the systems this rank owns (no data-path exchange)
    and the whole job's unit count (systems per bench step)."""
    from stokesdt_b200 import workloads as wl
    return wl.shard_systems(systems, world, rank), len(systems)


def run_b200_batch(args):
    """Config 4: 256 independent systems (N log-uniform in [500, 2e4], phi in
    [0.05, 0.3], grid and Ewald split per system by the autotuner, p = 6).
    One bench step = for every system: Update + one M.f + one 4-RHS block
    Lanczos.  Ranks own disjoint shards of the systems (weak in the sense
    that the job is fixed and split: strong scaling); value = systems/s of
    the whole job over the slowest rank."""
    import torch
    import stokesdt_b200 as sdt
    from stokesdt_b200 import workloads as wl

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    systems = wl.batch_systems()
    mine, total = batch_units(systems, world, rank)
    sy = [systems[i] for i in mine]
    npos = [s["npos"] for s in sy]
    pos = np.concatenate([wl.rsa_positions(s["npos"], s["box"], s["seed"]).reshape(-1) for s in sy])
    b = sdt.MobSpmeBatch(npos, np.ones(sum(npos)), [s["box"] for s in sy], [s["K"] for s in sy],
                         [s["xi"] for s in sy], [s["rmax"] for s in sy], porder=6, max_iters=100,
                         max_nrhs=4, tol=1e-6, reorth=True, lanes=8, device=local)
    tot = int(b.offsets[-1])
    rng = np.random.default_rng(41 + rank)
    d_pos = torch.tensor(pos, device=dev)
    d_F = torch.tensor(rng.standard_normal(tot), device=dev)
    d_V = torch.zeros(tot, dtype=torch.float64, device=dev)
    d_Z = torch.tensor(rng.standard_normal(4 * tot), device=dev)
    d_Y = torch.zeros(4 * tot, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)

    def step():
        b.update_device(d_pos.data_ptr())
        b.mulvec_device(1, 1.0, d_F.data_ptr(), 0.0, d_V.data_ptr())
        its = b.lanczos_device(4, d_Z.data_ptr(), d_Y.data_ptr())
        b.synchronize()
        return its

    if args.profile_case:
        # small case for ncu launch lists: an update and two 4-RHS packed products
        b.update_device(d_pos.data_ptr())
        for _ in range(2):
            b.mulvec_device(4, 1.0, d_Z.data_ptr(), 0.0, d_Y.data_ptr())
        b.synchronize()
        return

    def barrier():
        torch.cuda.synchronize(dev)
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(dev)

    for _ in range(args.warmup):
        step()
    barrier()
    sampler = ClockSampler(local)
    sampler.start()
    launches0 = sdt.kernel_launches()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    ev[0].record(stream)
    its = []
    for k in range(args.steps):
        its = step()                 # the lanes are synchronised inside
        ev[k + 1].record(stream)
    torch.cuda.synchronize(dev)
    barrier()
    clocks = sampler.stop()
    launches = sdt.kernel_launches() - launches0
    step_ms = [ev[k].elapsed_time(ev[k + 1]) for k in range(args.steps)]
    total_ms = max_over_ranks(dist, ev[0].elapsed_time(ev[-1]), dev)
    value = total * args.steps / (total_ms / 1e3)

    packed = b.packed
    # per-phase wall time of one more step (synchronised between phases)
    phase = {}
    barrier()
    t0 = time.perf_counter()
    b.update_device(d_pos.data_ptr())
    b.synchronize()
    t1 = time.perf_counter()
    b.mulvec_device(1, 1.0, d_F.data_ptr(), 0.0, d_V.data_ptr())
    b.synchronize()
    t2 = time.perf_counter()
    b.lanczos_device(4, d_Z.data_ptr(), d_Y.data_ptr())
    b.synchronize()
    t3 = time.perf_counter()
    phase = {"update": round(1e3 * (t1 - t0), 1), "mf_1rhs": round(1e3 * (t2 - t1), 1),
             "lanczos_4rhs": round(1e3 * (t3 - t2), 1)}
    log(f"config 4 phases (ms): {phase}")

    e2e = None
    if not args.no_e2e:
        hF = torch.tensor(d_F.cpu().numpy()).pin_memory().numpy()
        hV = torch.zeros(tot, dtype=torch.float64).pin_memory().numpy()
        hZ = torch.tensor(d_Z.cpu().numpy()).pin_memory().numpy()
        hY = torch.zeros(4 * tot, dtype=torch.float64).pin_memory().numpy()
        hp = torch.tensor(pos).pin_memory().numpy()
        barrier()
        h0, h1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ke = max(1, min(args.steps, 2))
        h0.record(stream)
        for _ in range(ke):
            b.Update(hp)
            b.MulVector(1, 1.0, hF, 0.0, hV)
            b.Lanczos(4, hZ, hY)
        h1.record(stream)
        torch.cuda.synchronize(dev)
        e_ms = max_over_ranks(dist, h0.elapsed_time(h1), dev)
        e2e = {"value": total * ke / (e_ms / 1e3), "unit": "systems/s",
               "h2d_bytes_per_step": 8 * (len(pos) + tot + 4 * tot),
               "d2h_bytes_per_step": 8 * (tot + 4 * tot), "steps": ke}

    # the same step with every system's own launches spread over the lanes,
    # then the plain per-system path: each system through the single-system
    # API (MobSpme + BrwnLanczos), one after the other
    def timed(fn, reps):
        barrier()
        t0 = time.perf_counter()
        for _ in range(reps):
            fn()
        torch.cuda.synchronize(dev)
        return (time.perf_counter() - t0) / reps

    lanes_rate = None
    if packed and not args.no_compare:
        b.set_packed(False)
        step()
        lanes_rate = len(mine) / timed(step, max(1, min(args.steps, 2)))
        b.set_packed(True)
    del b
    torch.cuda.empty_cache()
    plain_rate = None
    if not args.no_compare:
        engines = []
        for i, s in enumerate(sy):
            m = sdt.MobSpme(s["npos"], np.ones(s["npos"]), s["box"], s["xi"], s["rmax"], s["K"], 6, device=local)
            assert m.Init()
            m.set_stream(stream.cuda_stream)
            lz = sdt.BrwnLanczos(3 * s["npos"], 100, 4, 1e-6, device=local, reorth=True)
            assert lz.Init()
            lz.set_stream(stream.cuda_stream)
            engines.append((m, lz))
        off = np.concatenate([[0], np.cumsum([3 * s["npos"] for s in sy])])

        def plain_step():
            for i, (m, lz) in enumerate(engines):
                n3 = int(off[i + 1] - off[i])
                m.update_device(d_pos.data_ptr() + 8 * int(off[i]))
                m.mulvec_device(0, 1, 1.0, n3, d_F.data_ptr() + 8 * int(off[i]), 0.0, n3,
                                d_V.data_ptr() + 8 * int(off[i]))
                lz.compute_device(m, 4, n3, d_Z.data_ptr() + 32 * int(off[i]), n3,
                                  d_Y.data_ptr() + 32 * int(off[i]))

        plain_step()
        plain_rate = len(mine) / timed(plain_step, 1)
        del engines
    if rank == 0:
        lat = np.array(step_ms)
        out = {
            "metric": "systems/s (config 4: Update + M.f + 4-RHS Lanczos per system)",
            "value": round(value, 3), "unit": "systems/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(total_ms / args.steps, 3), "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
            "config": {"workload": "256 systems, N log-uniform [500, 20000], phi U[0.05, 0.3], K per system "
                                   "(autotuned, 64/128), p=6, 1 M.f + 4-RHS Lanczos tol 1e-6 each",
                       "systems": total, "particles": int(sum(s["npos"] for s in systems)),
                       "mode": "packed launches over all systems" if packed else "lanes",
                       "lanes_per_gpu": 8, "parallelism": f"systems sharded over {world} GPU(s)",
                       "l2": "no flush: per-system grids and pair lists total ~30 GB"},
            "phase_ms_rank0": phase,
            "lanes_mode_systems_per_s_rank0": None if lanes_rate is None else round(lanes_rate, 3),
            "plain_per_system_systems_per_s_rank0": None if plain_rate is None else round(plain_rate, 3),
            "packed_over_plain": (None if plain_rate is None else
                                  round(len(mine) * args.steps / (total_ms / 1e3) / plain_rate, 3)),
            "e2e": e2e, "gpu_launches": int(launches), "clocks": clocks,
            "latency_ms": {"p50": round(float(np.percentile(lat, 50)), 3),
                           "p99": round(float(np.percentile(lat, 99)), 3)},
            "lanczos_iters_median": float(np.median([i for i in its if i > 0])) if its else None,
        }
        print(json.dumps(out))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def serve_requests(nsys: int, nreq: int, rate: float, seed: int):
    """Config 5 request list: Poisson arrivals at `rate` per second, each a
    mobility apply (kind 0) or a Brownian step (kind 1) with k in {1, 4, 16}
    on one of nsys systems."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, nreq))
    return [(float(t[i]), int(rng.integers(nsys)), int(rng.integers(2)), int(rng.choice([1, 4, 16])))
            for i in range(nreq)]


def serve_systems(world: int):
    """Config 5 systems, 12 per rank: N log-uniform in [1e3, 1e5], phi
    uniform in [0.05, 0.3], grid / xi / rmax from the autotuner (K <= 256)."""
    from stokesdt_b200 import workloads as wl
    rng = np.random.default_rng(41)
    nsys = 12 * world
    npos = np.exp(rng.uniform(np.log(1e3), np.log(1e5), nsys)).astype(int)
    phis = rng.uniform(0.05, 0.3, nsys)
    systems = []
    for s in range(nsys):
        K, xi, rmax = wl.autotune_system(int(npos[s]), float(phis[s]), kmax=256)
        L = wl.box_for(int(npos[s]), float(phis[s]))
        systems.append(dict(npos=int(npos[s]), box=L, K=K, xi=xi, rmax=rmax, seed=4100 + s))
    return systems


def rank_share(reqs, mine):
    """The requests of `reqs` whose system this rank serves."""
    own = set(mine)
    return [r for r in reqs if r[1] in own]


def gather_all(dist, vals, world: int):
    """Every rank's list of values, concatenated in rank order."""
    if dist is None:
        return list(vals)
    parts = [None] * world
    dist.all_gather_object(parts, list(vals))
    return [v for p in parts for v in p]


def run_b200_serve(args):
    """Config 5: a served request stream (sdt_serve_*): systems with N
    log-uniform in [1e3, 1e5] and phi uniform in [0.05, 0.3] are registered
    once (device-resident, admitted by HBM budget); requests arrive as a
    Poisson stream at swept rates, plus one burst (every request at t = 0)
    that measures capacity.  Under torchrun the systems are split over the
    ranks by cost (largest first onto the least-loaded rank) and each rank
    serves the requests on its own systems: no data is exchanged, NCCL carries
    only the barrier and the max over ranks.  A rate's span runs from the
    common start to the slowest rank's last completion; throughput = all
    ranks' requests / that span.  Also reported: p50/p99 latency over all
    requests, the continuous-batching counts, and (rank 0) the plain
    per-request path (engine built, updated, used and released per request,
    one at a time) on the same requests."""
    import torch
    import stokesdt_b200 as sdt
    from stokesdt_b200 import workloads as wl

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)
    systems = serve_systems(world)
    nsys = len(systems)
    mine = wl.shard_systems(systems, world, rank)
    srv = sdt.MobilityServer(device=local, hbm_budget_bytes=120e9, lanes=4,
                             max_npos=max(systems[s]["npos"] for s in mine), max_iters=100, max_nrhs=16, tol=1e-6)
    ids, pos, inputs = {}, {}, {}
    for s in mine:
        sd = systems[s]
        pos[s] = wl.rsa_positions(sd["npos"], sd["box"], sd["seed"]).reshape(-1)
        ids[s] = srv.register(sd["npos"], np.ones(sd["npos"]), sd["box"], sd["K"], sd["xi"], sd["rmax"], 6, pos[s])
        inputs[s] = np.random.default_rng(s).standard_normal((16, 3 * sd["npos"]))

    def serve(reqs):
        """This rank's share of `reqs`, submitted at their arrival times from
        the common start; returns (latencies, seconds to the last completion)."""
        outs, tickets = [], []
        if dist is not None:
            dist.barrier()
        t0 = time.perf_counter()
        for (ta, s, kind, k) in rank_share(reqs, mine):
            dt = ta - (time.perf_counter() - t0)
            if dt > 0:
                time.sleep(dt)
            x = np.ascontiguousarray(inputs[s][:k])
            out = np.zeros_like(x)
            outs.append(out)
            tickets.append(srv.submit(ids[s], kind, k, x, out))
        lat = [srv.wait(t) for t in tickets]
        return lat, time.perf_counter() - t0

    # warm-up: every system once with each kind
    nwarm = max(1, args.warmup // 3)
    for _ in range(nwarm):
        serve([(0.0, s, kind, 4) for s in range(nsys) for kind in (0, 1)])
    launches0 = sdt.kernel_launches()
    st0 = srv.stats()
    sampler = ClockSampler(local)
    sampler.start()
    per_rate = []
    nreq = max(20, 10 * args.steps) * world
    for rate in (5.0 * world, 20.0 * world, 80.0 * world, None):
        if rate is None:
            reqs = [(0.0, s, kind, k) for (_, s, kind, k) in serve_requests(nsys, nreq, 1.0, seed=99)]
        else:
            reqs = serve_requests(nsys, nreq, rate, seed=int(rate))
        st_a = srv.stats()
        lat, span = serve(reqs)
        st_b = srv.stats()
        span = max_over_ranks(dist, span, dev)
        lat = gather_all(dist, lat, world)
        nb = st_b["batches"] - st_a["batches"]
        nbr = st_b["batched_requests"] - st_a["batched_requests"]
        per_rate.append({"offered_per_s": rate if rate is not None else "burst", "requests": len(reqs),
                         "throughput_per_s": round(len(reqs) / span, 3),
                         "p50_ms": round(float(np.percentile(lat, 50)), 3),
                         "p99_ms": round(float(np.percentile(lat, 99)), 3),
                         "batches_rank0": nb, "requests_per_batch_rank0": round(nbr / nb, 3) if nb else None})
        if rank == 0:
            log(f"rate {rate}: {per_rate[-1]}")
    clocks = sampler.stop()
    launches = sdt.kernel_launches() - launches0
    st1 = srv.stats()
    srv.close()

    # plain per-request path (rank 0, its own systems) on the first requests of the lowest rate
    plain_lat = []
    if rank == 0:
        for (_, s, kind, k) in serve_requests(nsys, 4 * nreq, 5.0, seed=5):
            if s not in ids:
                continue
            if len(plain_lat) == 24:
                break
            sd = systems[s]
            t0 = time.perf_counter()
            m = sdt.MobSpme(sd["npos"], np.ones(sd["npos"]), sd["box"], sd["xi"], sd["rmax"], sd["K"], 6,
                            device=local)
            assert m.Init()
            m.Update(pos[s])
            n3 = 3 * sd["npos"]
            x = np.ascontiguousarray(inputs[s][:k])
            out = np.zeros_like(x)
            if kind == 0:
                m.MulVector(k, 1.0, n3, x, 0.0, n3, out)
            else:
                lz = sdt.BrwnLanczos(n3, 100, 16, 1e-6, device=local, reorth=True)
                assert lz.Init()
                lz.Compute(m, k, n3, x, n3, out)
                del lz
            del m
            plain_lat.append(1e3 * (time.perf_counter() - t0))
    if rank == 0:
        best = max(per_rate, key=lambda r: r["throughput_per_s"])
        out = {
            "metric": "served requests/s (config 5) and p50/p99 latency", "value": best["throughput_per_s"],
            "unit": "requests/s", "n_gpus": world, "steps": nreq, "warmup": 2 * nsys * nwarm,
            "ms_per_step": round(1e3 / best["throughput_per_s"], 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
            "config": {"workload": "Poisson request stream: mobility apply or Brownian step, k in {1,4,16}, "
                                   f"{nsys} systems (12 per GPU) N log-uniform [1e3, 1e5], phi U[0.05, 0.3], "
                                   "p=6, tol 1e-6; offered rates 5/20/80 per s per GPU and a burst",
                       "lanes": 4, "hbm_budget_gb": 120,
                       "systems_rank0": [(systems[s]["npos"], systems[s]["K"]) for s in mine],
                       "parallelism": f"systems sharded over {world} GPU(s) by cost, no data exchange",
                       "l2": "no flush: systems' grids exceed the 126 MB L2"},
            "per_rate": per_rate,
            "batching_rank0": {"batch_lanes": st1["batch_lanes"], "batches": st1["batches"] - st0["batches"],
                               "batched_requests": st1["batched_requests"] - st0["batched_requests"],
                               "completed": st1["completed"] - st0["completed"]},
            "plain_per_request_path": {"requests": len(plain_lat),
                                       "p50_ms": round(float(np.percentile(plain_lat, 50)), 3),
                                       "p99_ms": round(float(np.percentile(plain_lat, 99)), 3),
                                       "throughput_per_s": round(1e3 * len(plain_lat) / sum(plain_lat), 3)},
            "e2e": {"value": best["throughput_per_s"], "unit": "requests/s",
                    "note": "host-pointer requests: every request's inputs are copied in and results out"},
            "gpu_launches": int(launches), "clocks": clocks,
        }
        print(json.dumps(out))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def main():
    args = parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        from stokesdt_b200 import workloads as wl
        if args.workload == "cfg4":
            run_b200_batch(args)
            return
        if args.workload == "cfg5":
            run_b200_serve(args)
            return
        w = wl.WORKLOADS[args.workload]
        if w.nsteps > 0:
            run_b200_traj(args, w)
            return
        out = run_b200(args)
        if out is None:
            return
        world = int(os.environ.get("WORLD_SIZE", "1"))
        if world == 1 and args.workload == "cfg2" and not args.no_other_configs and not args.profile_case:
            # the config-2 engines are gone with run_b200; give their memory back first
            import gc
            import torch
            gc.collect()
            torch.cuda.empty_cache()
            out["other_configs"] = run_other_configs()
        print(json.dumps(out))


if __name__ == "__main__":
    main()
