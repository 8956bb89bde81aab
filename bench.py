"""Benchmark: KKT solves/s of the block-iLDL^T + SQMR path on B200.

Workload (default --config scale): K = [[H + 1e-8 I, A'], [A, -1e-8 I]] with
n = 200000, m = 100000, 6 nonzeros per column of A (3 in a band of half-width
32 around floor(j m / n), 3 uniform), H log-uniform in [1e-6, 1e6],
contiguous 32-row blocks, Bunch-Kaufman pivoting, level-0 fill,
fill_factor 1, threshold 0; one N(0,1) right-hand side; SQMR with tol 1e-8
and max_it 1000 (the driver's settings, apps/block_ildlt/block_ildlt_invariants.h:186-187).
The sparsity pattern's symbolic analysis is done once (as for a stream of
IPM iterations on one pattern); a step is one numeric factorization plus one
SQMR solve with the values resident in HBM.  L2 (126 MB) is flushed before
every step outside the timed events (a 512 MB write, then a 512 MB read that
pushes the written lines back to HBM).

`e2e` times the same step through the public C ABI with host buffers: K's
values and b copied host -> device from pinned memory, the factor and the
solve, and x copied device -> host, inside the timed region.

`--impl reference` times the CPU restatement of the reference's path (the
reference has no CPU numeric path; its host symbolic phase and GPU kernels
are restated in oracle/) on the same workload, every step whole: factor and
the complete SQMR solve on all host threads.

Every line states how the solves ended: `converged` (true relres <= 1e-8)
and `stop` ("tol" or "max_it").  On the scale workload (late-IPM H spanning
1e-6..1e6) block-iLDL(0) + SQMR stops at max_it with true relres ~1.45 --
culip's own GPU build does the same on this input -- so there the value is
the rate of max_it-capped solves.

Multi-GPU: independent replicas (one KKT system per rank, no collective on
the data path); value = solves of all ranks / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# a solve stops at relres 1e-8 or at max_it; every line says which (converged, stop)
METRIC = "KKT solves/s (block-iLDLt + SQMR to tol 1e-8 or max_it, FP64 plain path)"
UNIT = "solves/s"


def _parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="culipx", choices=["culipx", "reference"])
    ap.add_argument("--config", default="scale", choices=["small", "scale", "mixed", "batch", "served", "spmv", "schur"])
    ap.add_argument("--spmv-workload", default="mixed", choices=["small", "scale", "mixed"],
                    help="--config spmv: the KKT matrix whose product is timed")
    ap.add_argument("--spmv-format", default="sell", choices=["csr", "sell"],
                    help="--config spmv: the CSR arrays or the SELL-32 copy (culipx_csr_set_format)")
    ap.add_argument("--rate", type=float, default=2000.0, help="--config served: arrivals per second")
    ap.add_argument("--duration", type=float, default=0.25, help="--config served: seconds of arrivals")
    ap.add_argument("--patterns", type=int, default=64, help="--config served: sparsity patterns")
    ap.add_argument("--plain", action="store_true",
                    help="--config served: the same requests through the plain FP64 path, one after another (FP64 "
                         "factor, one single-right-hand-side solve at a time, no server)")
    ap.add_argument("--precision", default="f32", choices=["f32", "f64"],
                    help="--config served: factor precision (f32: FP32 factor and applies, FP64 SQMR)")
    ap.add_argument("--refine", type=int, default=0,
                    help="--config served: FP64 refinement corrections per right-hand side (0: none)")
    ap.add_argument("--large-rows", type=int, default=131072,
                    help="--config served: patterns with N >= this use the whole-GPU solver")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--max-it", type=int, default=1000, help="SQMR iteration cap (1000 = the driver's setting)")
    ap.add_argument("--batch", type=int, default=512, help="systems in --config batch")
    ap.add_argument("--max-refine", type=int, default=10, help="--config mixed / batch: refinement corrections")
    ap.add_argument("--tune", type=int, default=1, help="--config batch: 1 = block size from culipx_tune_kkt_block")
    return ap.parse_args()


def _workload(name):
    import culip_b200 as cb

    cfg = dict(cb.KKT_CONFIGS[name])
    rp, ci, v = cb.kkt_generate(cfg["n"], cfg["m"], cfg["nnz_per_col"], cfg["band_half"], cfg["hmin"], cfg["hmax"])
    bs = cb.kkt_blocking(cfg["n"], cfg["m"], cfg["block"])
    b = cb.normal_vector(cb.SEED + 1, len(rp) - 1)
    return cfg, rp, ci, v, bs, b


def _config_dict(name, cfg, nnz, extra=None, solve="SQMR tol 1e-8 max_it 1000, 1 RHS"):
    d = {"workload": f"KKT {name}: n={cfg['n']} m={cfg['m']} N={cfg['n'] + cfg['m']} nnz_K={nnz}, "
                     f"A {cfg['nnz_per_col']}/col (band_half={cfg['band_half']}), H log-U[{cfg['hmin']:g},{cfg['hmax']:g}], "
                     f"blocks {cfg['block']}, BK, fill 0, {solve}",
         "pattern_reuse": "symbolic analysis once, numeric factor + solve per step",
         "l2": L2Flush.NOTE}
    if extra:
        d.update(extra)
    return d


class L2Flush:
    """Evicts L2 (126 MB) between timed steps, outside the timed events: a
    512 MB buffer is written, then a second 512 MB buffer is read, so the
    written lines are already back in HBM when the next step starts (a write
    alone leaves up to 126 MB of dirty lines whose write-back would be
    charged to the timed kernel)."""

    NOTE = "flushed before every step (512 MB write + 512 MB read outside the timed events)"

    def __init__(self):
        import torch

        self.w = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
        self.r = torch.ones(512 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def fill_(self, v):
        self.w.fill_(v)
        self.r.max()


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    def __init__(self, device=0):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def _host_threads():
    """Host threads this process may use (its CPU affinity)."""
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def reduce_max(value, dist=None):
    """The maximum of a float over all ranks (replicas: the job's time is its
    slowest rank's); NCCL reduces a CUDA tensor, gloo a CPU one."""
    if dist is None or not dist.is_initialized():
        return float(value)
    import torch

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(world, units_per_rank, max_seconds):
    """Whole-job throughput of replicas: every rank processed units_per_rank
    units; the job took as long as its slowest rank."""
    return world * units_per_rank / max_seconds


def _dist():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def run_culipx(args):
    import torch

    import culip_b200 as cb
    from culip_b200 import _capi as capi

    world, rank, local = _dist()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    cfg, rp, ci, v, bs, b = _workload(args.config)
    N = len(rp) - 1
    nnz = len(ci)
    stream = torch.cuda.current_stream()
    h = cb.Handle(local, stream)
    P = cb.Pattern(h, rp, ci, bs, 0, 1.0, cb.F64)
    F = cb.Factor(P)
    d_rp = torch.from_numpy(rp).cuda()
    d_ci = torch.from_numpy(ci).cuda()
    d_v = torch.from_numpy(v).cuda()
    d_b = torch.from_numpy(b).cuda()
    d_x = torch.zeros(N, dtype=torch.float64, device="cuda")
    A = cb.CsrOperator(h, d_rp, d_ci, d_v)
    flush = L2Flush()

    iters_seen = []
    sq_ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]

    def step(i=None):
        F.compute_graph(d_v, cb.PIV_BK, 0.0)  # the factorization's ~31 kernels as one graph launch
        if i is not None:
            sq_ev[i][0].record(stream)
        res, its, st = cb.sqmr_solve(h, A, F, d_b, d_x, 1e-8, args.max_it)
        if i is not None:
            sq_ev[i][1].record(stream)
        iters_seen.append(its)
        return res, its

    for _ in range(args.warmup):
        flush.fill_(1.0)
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    h.launch_count(reset=True)
    clocks = ClockSampler(local)
    clocks.start()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    torch.cuda.synchronize()
    for i in range(args.steps):
        flush.fill_(float(i))
        evs[i][0].record(stream)
        step(i)
        evs[i][1].record(stream)
    torch.cuda.synchronize()
    ck = clocks.stop()
    launches = h.launch_count(reset=True)
    step_ms = [a.elapsed_time(b2) for a, b2 in evs]
    total_ms = reduce_max(float(np.sum(step_ms)), dist)
    if dist:
        dist.barrier()

    # accuracy of the last step
    x = d_x.cpu().numpy()
    import scipy.sparse as sp

    K = sp.csr_matrix((v, ci, rp), shape=(N, N))
    relres = float(np.linalg.norm(b - K @ x) / np.linalg.norm(b))

    # roofline of the dominant kernel, the persistent SQMR launch (one per solve)
    sq_ms = float(np.mean([a0.elapsed_time(b0) for a0, b0 in sq_ev]))
    roof = sqmr_roofline(F.info(), N, nnz, int(np.median(iters_seen)), sq_ms)

    # e2e through the public API with host buffers
    hv = torch.from_numpy(v).pin_memory()
    hb = torch.from_numpy(b).pin_memory()
    hx = torch.empty(N, dtype=torch.float64).pin_memory()
    d_v2 = torch.empty_like(d_v)
    d_b2 = torch.empty_like(d_b)
    A2 = cb.CsrOperator(h, d_rp, d_ci, d_v2)
    e2e_steps = max(2, min(args.steps, 5))
    d_v2.copy_(d_v)
    F.compute_graph(d_v2, cb.PIV_BK, 0.0)  # capture for this buffer before the timed region
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    e_ms = []
    for i in range(e2e_steps):
        flush.fill_(float(i))
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        d_v2.copy_(hv, non_blocking=True)
        d_b2.copy_(hb, non_blocking=True)
        F.compute_graph(d_v2, cb.PIV_BK, 0.0)
        cb.sqmr_solve(h, A2, F, d_b2, d_x, 1e-8, args.max_it)
        hx.copy_(d_x, non_blocking=True)
        e1.record(stream)
        torch.cuda.synchronize()
        e_ms.append(e0.elapsed_time(e1))
    e2e_total = reduce_max(float(np.sum(e_ms)), dist)

    fac_ms, fac_launches = F.stats()
    value = job_rate(world, args.steps, total_ms / 1e3)
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded KKT generator)",
        "config": _config_dict(args.config, cfg, nnz, {"parallelism": f"replicas x{world} (independent KKT systems)",
                                                        "max_it": args.max_it}),
        "sqmr_iterations": int(np.median(iters_seen)) if iters_seen else None,
        "true_relres": relres,
        "converged": relres <= 1e-8,
        "stop": "tol" if iters_seen and int(np.median(iters_seen)) < args.max_it else "max_it",
        "factor_ms": fac_ms,
        "gpu_launches": int(launches),
        "clocks": ck,
        "e2e": {"value": job_rate(world, e2e_steps, e2e_total / 1e3), "unit": UNIT,
                "h2d_bytes_per_step": int(nnz * 8 + N * 8), "d2h_bytes_per_step": int(N * 8)},
        "roofline": roof,
        "spmv": spmv_formats(h, d_rp, d_ci, d_v, N, nnz, flush, stream),
        "sweeps": sweep_roofline(F, N, flush, stream),
    }
    if args.config == "small":
        # the small workload reaches a true relres of 1e-8 with FP64 iterative
        # refinement around SQMR (its quasi-residual stop alone leaves ~5e-6):
        # factor (graph) + culipx_sqmr_refine per step, inner SQMR tol 1e-6
        r_ms, r_out = [], None
        for i in range(args.warmup + args.steps):
            flush.fill_(float(i))
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            F.compute_graph(d_v, cb.PIV_BK, 0.0)
            r_out = cb.sqmr_refine(h, A, F, d_b, d_x, 1e-8, 1e-6, args.max_it, 10)
            e1.record(stream)
            torch.cuda.synchronize()
            if i >= args.warmup:
                r_ms.append(e0.elapsed_time(e1))
        xr = d_x.cpu().numpy()
        rel_r = float(np.linalg.norm(b - K @ xr) / np.linalg.norm(b))
        out["refined"] = {"what": "factor + FP64 refinement around SQMR (inner tol 1e-6) to true relres 1e-8",
                          "value": args.steps / (float(np.sum(r_ms)) / 1e3), "unit": UNIT,
                          "ms_per_step": float(np.mean(r_ms)), "true_relres": rel_r, "converged": rel_r <= 1e-8,
                          "sqmr_iterations": int(r_out[1]), "corrections": int(r_out[2]),
                          "status": capi.STATUS_NAMES.get(int(r_out[3]), int(r_out[3]))}
    if rank == 0 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(args.config, rp, ci, v, bs, b, args.max_it)
    if dist:
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out), flush=True)


def sqmr_roofline(info, N, nnz, its, launch_ms, nr=1, kernel="k_sqmr_persistent<double> (one cooperative launch per solve)",
                  profile="sqmr_persistent_scale.txt"):
    """Algorithmic bytes of one persistent SQMR launch (init, its iterations,
    final solve) over its CUDA-event duration.  Per iteration:
      B_spmv = nnz_K (8 + 4) + 4 (N + 1) + 8 N (x) + 8 N (y)
      B_tri  = nnz_U (s + 4) + 4 (N + 1) + s * (upper-triangle entries of the
               non-identity pivot tiles) + 2 * 8 N
      B_D    = 3 N s + 2 * 8 N
      B_iter = B_spmv + 2 B_tri + 2 B_D + 11 * 8 N
    and the launch adds B_spmv + 4 B_tri for the initial sweeps and the final
    x = P U^-1 D^-1 x~.  With nr right-hand sides in one launch the matrix and
    factor terms are read once and every 8 N vector term counts nr times.
    traffic: DRAM bytes per iteration from the ncu summary under profiles/,
    times the iterations."""
    s = info["value_bytes"]
    b_spmv = nnz * 12 + 4 * (N + 1) + 16 * N * nr
    b_tri = info["u_nnz"] * (s + 4) + 4 * (N + 1) + s * info["tile_entries"] + 16 * N * nr
    b_d = 3 * N * s + 16 * N * nr
    b_iter = b_spmv + 2 * b_tri + 2 * b_d + 11 * 8 * N * nr
    b_launch = its * b_iter + b_spmv + 4 * b_tri
    achieved = b_launch / (launch_ms * 1e-3) / 1e9
    peak = _peak_hbm()
    traffic = None
    prof = os.path.join(ROOT, "profiles", profile)
    if os.path.exists(prof):
        for ln in open(prof):
            if ln.startswith("dram_bytes_per_iteration"):
                traffic = float(ln.split("=")[1]) * its
    return {"kernel": kernel, "bound": "hbm",
            "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
            "traffic_source": f"ncu dram__bytes_read.sum + dram__bytes_write.sum per iteration of this kernel, "
                              f"from profiles/{profile} (a separate capture, not this run), times the iterations",
            "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)",
            "algorithmic_bytes": int(b_launch), "bytes_per_iteration": int(b_iter), "iterations": its,
            "avg_launch_ms": launch_ms, "us_per_iteration": launch_ms * 1e3 / max(its, 1)}


def sweep_roofline(F, N, flush, stream, reps=10, precision_bytes=8):
    """The standalone triangular solves (culipx_prec_apply; the reference's
    solve_left / solve_right), L2 flushed before every call (outside the
    events): LEFT = x = U'^-1 P' b, RIGHT = x = P U^-1 b, one launch per level
    with the pivot permutation folded into the sweeps.
    Algorithmic bytes: B_tri = nnz_U (s + 4) + 4 (N + 1) + s * (upper-triangle
    entries of the non-identity pivot tiles) + 2 s N (read b, write x), plus
    the permutation (4 N)."""
    import torch

    import culip_b200 as cb

    info = F.info()
    s = info["value_bytes"]
    dt = torch.float64 if s == 8 else torch.float32
    b = torch.linspace(-1.0, 1.0, N, dtype=dt, device="cuda")
    x = torch.zeros_like(b)
    b_tri = info["u_nnz"] * (s + 4) + 4 * (N + 1) + s * info["tile_entries"] + 2 * s * N
    peak = _peak_hbm()
    out = {}
    for name, stage, extra in (("u_transpose_sweep (LEFT)", cb.LEFT, 4 * N), ("u_sweep (RIGHT)", cb.RIGHT, 4 * N)):
        for _ in range(3):
            F.apply(stage, b, x)
        ms = []
        for i in range(reps):
            flush.fill_(float(i))
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            F.apply(stage, b, x)
            e1.record(stream)
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1))
        t = float(np.mean(ms))
        byt = b_tri + extra
        out[name] = {"achieved": byt / (t * 1e-3) / 1e9, "frac": byt / (t * 1e-3) / 1e9 / peak,
                     "avg_us": t * 1e3, "algorithmic_bytes": int(byt)}
    out.update({"unit": "GB/s", "peak": peak, "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)",
                "kernels": "k_sweep_level per level (permutation folded in)",
                "l2": "flushed before every call"})
    return out


def spmv_formats(h, d_rp, d_ci, d_v, N, nnz, flush, stream, reps=20):
    """spmv_roofline for the CSR arrays and for the SELL-32 copy
    (culipx_csr_set_format), each on its own operator."""
    import culip_b200 as cb

    out = {}
    for name, fmt in (("csr", cb.FMT_CSR), ("sell", cb.FMT_SELL)):
        B = cb.CsrOperator(h, d_rp, d_ci, d_v)
        if fmt != cb.FMT_CSR:
            B.set_format(fmt)
        out[name] = spmv_roofline(B, N, nnz, flush, stream, reps,
                                  kernel="k_sell_spmv<double>" if fmt == cb.FMT_SELL else "k_csr_spmv_rows<double>")
    best = max(out, key=lambda k: out[k]["achieved"])
    res = dict(out[best])
    res["format"] = best
    res["formats"] = {k: {"achieved": o["achieved"], "frac": o["frac"], "avg_launch_us": o["avg_launch_us"]}
                      for k, o in out.items()}
    return res


def spmv_roofline(A, N, nnz, flush, stream, reps=20, kernel="k_csr_spmv_rows<double>"):
    """Standalone y = K x (culipx_spmv, FP64, beta = 0) with L2 flushed before
    every launch (outside the events): algorithmic bytes
    B_spmv = nnz_K (8 + 4) + 4 (N + 1) + 8 N (x) + 8 N (y) over the mean
    CUDA-event duration."""
    import torch

    x = torch.linspace(-1.0, 1.0, N, dtype=torch.float64, device="cuda")
    y = torch.zeros(N, dtype=torch.float64, device="cuda")
    for _ in range(3):
        A.spmv(x, y)
    ms = []
    for i in range(reps):
        flush.fill_(float(i))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        A.spmv(x, y)
        e1.record(stream)
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    t = float(np.mean(ms))
    b = nnz * 12 + 4 * (N + 1) + 16 * N
    peak = _peak_hbm()
    return {"kernel": f"{kernel} (culipx_spmv, L2 flushed before each launch)", "achieved": b / (t * 1e-3) / 1e9,
            "peak": peak, "unit": "GB/s", "frac": b / (t * 1e-3) / 1e9 / peak, "algorithmic_bytes": int(b),
            "avg_launch_us": t * 1e3, "launches": reps}


def _peak_hbm():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"])
    except Exception:
        return 6650.0


def cpu_baseline(name, rp, ci, v, bs, b, max_it):
    """The oracle (CPU restatement of the reference's path) on all host
    threads: one complete step, numeric factor (block rows of a level in
    parallel) plus the full SQMR solve (tol 1e-8, max_it), timed whole.  The
    symbolic analysis is cached per pattern, as on the GPU side."""
    import oracle

    cores = oracle.set_threads(_host_threads())
    S = oracle.Sym(rp, ci, bs, 0, 1.0)
    t0 = time.perf_counter()
    F = S.factor(v)
    t1 = time.perf_counter()
    _, _, its = oracle.sqmr(rp, ci, v, b, F, 1e-8, max_it)
    t2 = time.perf_counter()
    return {"value": 1.0 / (t2 - t0), "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"one full step: oracle factor {t1 - t0:.2f}s + SQMR {its} iterations {t2 - t1:.2f}s "
                      f"(plain loops, no BLAS)"}


def run_reference_spmv(args):
    """The CPU restatement's y = K x (CSR rows spread over the host threads) on the same
    matrix; value = algorithmic GB/s as in --config spmv."""
    import oracle

    cores = oracle.set_threads(_host_threads())

    cfg, rp, ci, v, bs, _ = _workload(args.spmv_workload)
    N, nnz = len(rp) - 1, len(ci)
    x = np.linspace(-1.0, 1.0, N)
    ms = []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        oracle.spmv(rp, ci, v, x)
        if i >= args.warmup:
            ms.append((time.perf_counter() - t0) * 1e3)
    t = float(np.mean(ms))
    b = nnz * 12 + 4 * (N + 1) + 16 * N
    gbs = b / (t * 1e-3) / 1e9
    out = {"metric": "SpMV HBM GB/s (culipx_spmv, FP64 CSR, y = K x)", "value": gbs, "unit": "GB/s", "n_gpus": 1,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": t, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded KKT generator)", "impl": "reference",
           "config": _config_dict(args.spmv_workload, cfg, nnz, {"parallelism": f"{cores} CPU threads"}, solve="y = K x only"),
           "cpu_baseline": {"value": gbs, "unit": "GB/s", "cores": cores, "kind": "port",
                            "sample": "oracle CSR product (rows over the host threads), whole matrix per step"},
           "e2e": {"value": gbs, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def run_reference_batch(args):
    """The CPU restatement on the batched workload: each step solves one
    system of the 512 (a fixed spread sample, system 37 k mod 512 at step k)
    with the whole algorithm: FP64 factor (the restatement's SQMR takes an
    FP64 factor) and the same refinement loop (inner SQMR tol 1e-6, max_it,
    at most --max-refine corrections, true FP64 residual, target 1e-8);
    value = systems solved per second (the restatement's row-independent loops
    on all host threads)."""
    import oracle

    cores = oracle.set_threads(_host_threads())

    syst = batch_systems(args.batch)
    ms, its_all = [], []
    for i in range(args.warmup + args.steps):
        rp, ci, v, bs = syst[(37 * i) % len(syst)]
        N = len(rp) - 1
        b = __import__("culip_b200").normal_vector(__import__("culip_b200").SEED + 4000 + 100000 + (37 * i) % len(syst), N)
        t0 = time.perf_counter()
        F = oracle.Sym(rp, ci, bs, 0, 1.0).factor(v)
        x = np.zeros(N)
        r = b.copy()
        nb = float(np.linalg.norm(b))
        its = 0
        for _ in range(args.max_refine):
            if np.linalg.norm(r) <= 1e-8 * nb:
                break
            d, _, it = oracle.sqmr(rp, ci, v, r, F, 1e-6, args.max_it)
            its += it
            x += d
            r = b - oracle.spmv(rp, ci, v, x)
        if i >= args.warmup:
            ms.append((time.perf_counter() - t0) * 1e3)
            its_all.append(its)
    t = float(np.mean(ms))
    value = 1e3 / t
    out = {"metric": "KKT solves/s (batched uneven instances, FP32 factor + FP64 refinement to relres 1e-8)",
           "value": value, "unit": "solves/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": t, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic (seeded KKT generator)", "impl": "reference",
           "config": {"workload": f"{len(syst)} KKT systems, n U[500,20000], m=n/2, A 4-8/col (band_half=32), "
                                  f"H log-U[1e-4,1e4], blocks 32, BK, fill 0",
                      "solver": f"oracle FP64 factor + SQMR (inner tol 1e-6, max_it {args.max_it}) in the same "
                                f"refinement loop, at most {args.max_refine} corrections", "parallelism": f"{cores} CPU threads"},
           "cpu_baseline": {"value": value, "unit": "solves/s", "cores": cores, "kind": "port",
                            "sample": f"{args.steps} systems (37 k mod 512), each solved whole; median SQMR "
                                      f"iterations {int(np.median(its_all))}"},
           "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def run_reference_served(args):
    """The CPU restatement on the served stream's requests, one after another
    on the host (row-independent loops on all threads): each step takes the next request of the same arrival trace
    (pattern, 1-8 right-hand sides; the trace's first --warmup + --steps
    requests) and runs the oracle's factor plus, per right-hand side, a
    20-iteration SQMR sample scaled to max_it iterations (every right-hand
    side of this stream runs to max_it: none reaches 1e-8); value = requests
    per second."""
    import oracle

    cores = oracle.set_threads(_host_threads())

    import culip_b200 as cb

    seed_base = cb.SEED + 5000
    pats = served_workload(args.patterns, seed_base)
    rng = np.random.default_rng(seed_base + 999)
    reqs = []
    while len(reqs) < args.warmup + args.steps:
        rng.exponential(1.0 / args.rate)
        reqs.append((int(rng.integers(0, len(pats))), int(rng.integers(1, 9))))
    syms = {}
    ms = []
    sample_it = 20
    for i, (j, nrhs) in enumerate(reqs):
        rp, ci, v, bs, n = pats[j]
        N = len(rp) - 1
        if j not in syms:
            syms[j] = oracle.Sym(rp, ci, bs, 0, 1.0)  # the server analyses each pattern once
        t0 = time.perf_counter()
        F = syms[j].factor(v)
        t1 = time.perf_counter()
        solve = 0.0
        for k in range(nrhs):
            b = cb.normal_vector(seed_base + 7 * i + k, N)
            t2 = time.perf_counter()
            oracle.sqmr(rp, ci, v, b, F, 1e-8, sample_it)
            solve += (time.perf_counter() - t2) / sample_it * args.max_it
        if i >= args.warmup:
            ms.append(((t1 - t0) + solve) * 1e3)
    t = float(np.mean(ms))
    value = 1e3 / t
    out = {"metric": "KKT solves/s and p50/p99 latency (served IPM stream, FP64 plain method per request)",
           "value": value, "unit": "requests/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": t, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic (seeded KKT generator, Poisson arrivals)", "impl": "reference",
           "config": {"workload": f"{len(pats)} patterns, n log-U[1e3,5e5], m=n/2, A 6/col (band_half=32), "
                                  f"the served trace's requests, 1-8 RHS",
                      "solver": f"oracle factor + SQMR tol 1e-8, max_it {args.max_it}, requests one after another",
                      "parallelism": f"{cores} CPU threads"},
           "latency_ms": {"p50": float(np.percentile(ms, 50)), "p99": float(np.percentile(ms, 99))},
           "cpu_baseline": {"value": value, "unit": "requests/s", "cores": cores, "kind": "port",
                            "sample": f"{args.steps} requests of the trace: factor whole, SQMR {sample_it} "
                                      f"iterations per right-hand side scaled to {args.max_it}"},
           "e2e": {"value": value, "unit": "requests/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def run_reference(args):
    world, rank, _ = _dist()
    if rank != 0:
        return
    if args.config == "spmv":
        return run_reference_spmv(args)
    if args.config == "batch":
        return run_reference_batch(args)
    if args.config == "served":
        return run_reference_served(args)
    cfg, rp, ci, v, bs, b = _workload(args.config)
    import oracle

    cores = oracle.set_threads(_host_threads())
    S = oracle.Sym(rp, ci, bs, 0, 1.0)
    # one step = numeric factor + the complete SQMR solve, as on the GPU side
    ms, its_seen = [], []
    x = None
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        F = S.factor(v)
        x, _, it = oracle.sqmr(rp, ci, v, b, F, 1e-8, args.max_it)
        t1 = time.perf_counter()
        if i >= args.warmup:
            ms.append((t1 - t0) * 1e3)
            its_seen.append(it)
    total = float(np.sum(ms))
    value = args.steps / (total / 1e3)
    import scipy.sparse as sp

    N = len(rp) - 1
    relres = float(np.linalg.norm(b - sp.csr_matrix((v, ci, rp), shape=(N, N)) @ x) / np.linalg.norm(b))
    out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": total / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "f64", "data": "synthetic (seeded KKT generator)", "impl": "reference",
           "config": _config_dict(args.config, cfg, len(ci), {"parallelism": f"replicas x{world} (independent KKT systems)",
                                                             "max_it": args.max_it}),
           "sqmr_iterations": int(np.median(its_seen)), "true_relres": relres,
           "converged": relres <= 1e-8, "stop": "tol" if int(np.median(its_seen)) < args.max_it else "max_it",
           "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                            "sample": "every step timed whole: oracle factor (block rows of a level on all host "
                                      "threads) + the complete SQMR solve (plain loops, no BLAS)"},
           "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def run_mixed(args):
    """Mixed precision with several right-hand sides (n = 1e6, m = 5e5, 4
    N(0,1) right-hand sides): FP32 factor and preconditioner applies, FP64
    SQMR recurrence, FP64 true residual and refinement to relres 1e-10, the 4
    right-hand sides solved together in multi-RHS launches.  A step = FP32
    factor + the refined solve of all 4; value = right-hand sides solved per
    second.  The error is stated against the FP64 path (FP64 factor, plain
    SQMR on the same right-hand sides)."""
    import torch

    import culip_b200 as cb

    world, rank, local = _dist()
    torch.cuda.set_device(local)
    nr = 4
    cfg, rp, ci, v, bs, _ = _workload("mixed")
    N, nnz = len(rp) - 1, len(ci)
    Bh = np.stack([cb.normal_vector(cb.SEED + 1 + j, N) for j in range(nr)])
    stream = torch.cuda.current_stream()
    h = cb.Handle(local, stream)
    P = cb.Pattern(h, rp, ci, bs, 0, 1.0, cb.F32)
    F = cb.Factor(P)
    d_rp = torch.from_numpy(rp).cuda()
    d_ci = torch.from_numpy(ci).cuda()
    d_v = torch.from_numpy(v).cuda()
    d_v32 = d_v.float()
    d_B = torch.from_numpy(Bh).cuda()
    d_X = torch.zeros_like(d_B)
    A = cb.CsrOperator(h, d_rp, d_ci, d_v)
    flush = L2Flush()
    tol, inner_tol, inner_it, max_ref = 1e-10, 1e-6, args.max_it, args.max_refine
    stats = {}

    def step():
        F.compute_graph(d_v32, cb.PIV_BK, 0.0)
        rel, its, steps, st = cb.sqmr_refine_multi(h, A, F, d_B, d_X, tol, inner_tol, inner_it, max_ref)
        stats.update(rel=rel, its=its, steps=steps, st=st)

    for _ in range(args.warmup):
        flush.fill_(1.0)
        step()
    torch.cuda.synchronize()
    h.launch_count(reset=True)
    clocks = ClockSampler(local)
    clocks.start()
    ms = []
    for i in range(args.steps):
        flush.fill_(float(i))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        step()
        e1.record(stream)
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    ck = clocks.stop()
    launches = h.launch_count(reset=True)
    total_ms = float(np.sum(ms))
    fac_ms, _ = F.stats()
    Xm = d_X.cpu().numpy()

    # the multi-RHS launch alone, for the roofline: a fixed 200 iterations (tol 0)
    its_roof = 200
    R = torch.zeros_like(d_B)
    for _ in range(2):
        cb.sqmr_solve_multi(h, A, F, d_B, R, 0.0, its_roof)
    flush.fill_(2.0)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    cb.sqmr_solve_multi(h, A, F, d_B, R, 0.0, its_roof)
    e1.record(stream)
    torch.cuda.synchronize()
    roof = sqmr_roofline(F.info(), N, nnz, its_roof, e0.elapsed_time(e1), nr=nr,
                         kernel="k_sqmr_persistent<float, NR=4> (4 right-hand sides per cooperative launch)",
                         profile="sqmr_persistent_mixed.txt")

    # e2e: K's values and the 4 right-hand sides from pinned host memory, X back
    hv = torch.from_numpy(v).pin_memory()
    hB = torch.from_numpy(Bh).pin_memory()
    hX = torch.empty_like(hB).pin_memory()
    e_ms = []
    for i in range(max(2, min(args.steps, 3))):
        flush.fill_(float(i))
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        d_v.copy_(hv, non_blocking=True)
        d_B.copy_(hB, non_blocking=True)
        d_v32.copy_(d_v)
        step()
        hX.copy_(d_X, non_blocking=True)
        e1.record(stream)
        torch.cuda.synchronize()
        e_ms.append(e0.elapsed_time(e1))

    # the FP64 path on the same right-hand sides: FP64 factor, plain SQMR
    P64 = cb.Pattern(h, rp, ci, bs, 0, 1.0, cb.F64)
    F64 = cb.Factor(P64)
    F64.compute(d_v, None, cb.PIV_BK, 0.0)
    X64 = torch.zeros_like(d_B)
    _, its64, st64 = cb.sqmr_solve_multi(h, A, F64, d_B, X64, tol, args.max_it)
    X64 = X64.cpu().numpy()
    import scipy.sparse as sp

    K = sp.csr_matrix((v, ci, rp), shape=(N, N))
    rel_m = [float(np.linalg.norm(Bh[j] - K @ Xm[j]) / np.linalg.norm(Bh[j])) for j in range(nr)]
    rel_64 = [float(np.linalg.norm(Bh[j] - K @ X64[j]) / np.linalg.norm(Bh[j])) for j in range(nr)]
    err = [float(np.linalg.norm(Xm[j] - X64[j]) / max(np.linalg.norm(X64[j]), 1e-300)) for j in range(nr)]
    out = {
        "metric": "KKT right-hand sides solved/s (FP32 factor + FP64 refinement to relres 1e-10, 4 RHS per system)",
        "value": nr * args.steps / (total_ms / 1e3), "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 factor / f64 recurrence and refinement",
        "data": "synthetic (seeded KKT generator)",
        "config": _config_dict("mixed", cfg, nnz, {
            "solver": f"{nr} RHS in one multi-RHS SQMR launch per correction, inner tol {inner_tol:g} max_it "
                      f"{inner_it}, FP64 refinement to {tol:g}, at most {max_ref} corrections",
            "parallelism": "one GPU"}, solve=f"FP32 factor, {nr} N(0,1) RHS, relres 1e-10"),
        "true_relres": rel_m, "status": [int(t) for t in stats["st"]],
        "sqmr_iterations": [int(t) for t in stats["its"]], "corrections": [int(t) for t in stats["steps"]],
        "fp64_path": {"true_relres": rel_64, "sqmr_iterations": [int(t) for t in its64],
                      "status": [int(t) for t in st64]},
        "rel_error_vs_fp64_path": err,
        "factor_ms": fac_ms, "gpu_launches": int(launches), "clocks": ck,
        "e2e": {"value": nr * len(e_ms) / (float(np.sum(e_ms)) / 1e3), "unit": "solves/s",
                "h2d_bytes_per_step": int(nnz * 8 + nr * N * 8), "d2h_bytes_per_step": int(nr * N * 8)},
        "roofline": roof,
        "spmv": spmv_formats(h, d_rp, d_ci, d_v, N, nnz, flush, stream),
        "sweeps": sweep_roofline(F, N, flush, stream),
    }
    if rank == 0:
        print(json.dumps(out), flush=True)


def run_spmv(args):
    """y = K x alone (culipx_spmv, FP64, beta = 0) on a KKT matrix: a step is
    one product with L2 flushed before it; value = algorithmic HBM GB/s
    (nnz_K (8 + 4) + 4 (N + 1) + 8 N + 8 N bytes per product)."""
    import torch

    import culip_b200 as cb

    world, rank, local = _dist()
    torch.cuda.set_device(local)
    cfg, rp, ci, v, bs, _ = _workload(args.spmv_workload)
    N, nnz = len(rp) - 1, len(ci)
    stream = torch.cuda.current_stream()
    h = cb.Handle(local, stream)
    A = cb.CsrOperator(h, torch.from_numpy(rp).cuda(), torch.from_numpy(ci).cuda(), torch.from_numpy(v).cuda())
    kname = "k_csr_spmv_rows<double>"
    if args.spmv_format == "sell":
        A.set_format(cb.FMT_SELL)
        kname = "k_sell_spmv<double>"
    flush = L2Flush()
    x = torch.linspace(-1.0, 1.0, N, dtype=torch.float64, device="cuda")
    y = torch.zeros(N, dtype=torch.float64, device="cuda")
    for _ in range(args.warmup):
        flush.fill_(1.0)
        A.spmv(x, y)
    torch.cuda.synchronize()
    h.launch_count(reset=True)
    clocks = ClockSampler(local)
    clocks.start()
    ms = []
    for i in range(args.steps):
        flush.fill_(float(i))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        A.spmv(x, y)
        e1.record(stream)
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    ck = clocks.stop()
    launches = h.launch_count(reset=True)
    t = float(np.mean(ms))
    b = nnz * 12 + 4 * (N + 1) + 16 * N
    peak = _peak_hbm()
    gbs = b / (t * 1e-3) / 1e9
    # e2e: x from pinned host memory, y back
    hx = x.cpu().pin_memory()
    hy = torch.empty_like(hx).pin_memory()
    e_ms = []
    for i in range(max(3, min(args.steps, 10))):
        flush.fill_(float(i))
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        x.copy_(hx, non_blocking=True)
        A.spmv(x, y)
        hy.copy_(y, non_blocking=True)
        e1.record(stream)
        torch.cuda.synchronize()
        e_ms.append(e0.elapsed_time(e1))
    traffic = None
    prof = os.path.join(ROOT, "profiles", f"spmv_{'sell_' if args.spmv_format == 'sell' else ''}{args.spmv_workload}.txt")
    if os.path.exists(prof):
        for ln in open(prof):
            if ln.startswith("dram_bytes_per_launch"):
                traffic = float(ln.split("=")[1])
    out = {
        "metric": "SpMV HBM GB/s (culipx_spmv, FP64, y = K x)", "value": gbs, "format": args.spmv_format, "unit": "GB/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded KKT generator)",
        "config": _config_dict(args.spmv_workload, cfg, nnz, {"parallelism": "one GPU"}, solve="y = K x only"),
        "gpu_launches": int(launches), "clocks": ck,
        "e2e": {"value": b / (float(np.mean(e_ms)) * 1e-3) / 1e9, "unit": "GB/s", "h2d_bytes_per_step": int(8 * N),
                "d2h_bytes_per_step": int(8 * N)},
        "roofline": {"kernel": kname, "bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s",
                     "frac": gbs / peak, "traffic": traffic, "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)",
                     "algorithmic_bytes": int(b), "avg_launch_us": t * 1e3},
    }
    if rank == 0:
        print(json.dumps(out), flush=True)


def batch_systems(num=512, seed_base=None, block=32):
    """The batched workload: num KKT systems, system i from sub-seed
    SEED + 4000 + i, n uniform in [500, 20000], m = n // 2, A with 4-8
    nonzeros per column (half in a band of half-width 32, half uniform),
    H log-uniform in [1e-4, 1e4], delta = gamma = 1e-8, 32-row blocks."""
    import culip_b200 as cb

    rng = np.random.default_rng(cb.SEED + 4000)
    out = []
    for i in range(num):
        n = int(rng.integers(500, 20001))
        m = n // 2
        k = int(rng.integers(4, 9))
        rp, ci, v = cb.kkt_generate(n, m, k, 32, 1e-4, 1e4, seed=cb.SEED + 4000 + i)
        out.append((rp, ci, v, cb.kkt_blocking(n, m, block)))
    return out


def tune_batch_block(args, local, candidates=(8, 16, 24, 32), samples=(0, 128, 256, 384)):
    """Block size for the batched workload from culipx_tune_kkt_block on a
    sample of its systems (FP32 factor, tol 1e-8, max_it): the candidate
    whose solves met tol most often, then the least summed time (when none
    met it: the smallest residual estimates, the better start for refinement)."""
    import torch

    import culip_b200 as cb

    h = cb.Handle(local)
    rng = np.random.default_rng(cb.SEED + 4000)
    dims = [(int(rng.integers(500, 20001)), int(rng.integers(4, 9))) for _ in range(args.batch)]
    score = {c: [0, 0.0, 0.0] for c in candidates}
    for i in samples:
        if i >= args.batch:
            continue
        n, k = dims[i]
        rp, ci, v = cb.kkt_generate(n, n // 2, k, 32, 1e-4, 1e4, seed=cb.SEED + 4000 + i)
        b = cb.normal_vector(cb.SEED + 4000 + 100000 + i, len(rp) - 1)
        _, res = cb.tune_kkt_block(h, n, n // 2, rp, ci, torch.from_numpy(v).cuda(), torch.from_numpy(b).cuda(),
                                   cb.F32, candidates, 1e-8, args.max_it)
        for c, (ms, its, st, rr) in res.items():
            score[c][0] += int(st == 0)
            score[c][1] += ms
            score[c][2] += np.log10(max(rr, 1e-300))
    # most converged; then, if some converged, the least time, else the smallest residuals
    any_converged = max(score[c][0] for c in candidates) > 0
    best = min(candidates, key=lambda c: (-score[c][0], score[c][1] if any_converged else score[c][2]))
    return best, {str(c): {"converged": score[c][0], "ms": round(score[c][1], 3),
                           "mean_log10_residual": round(score[c][2] / len(samples), 3)} for c in candidates}


def run_batch(args):
    """Batched uneven instances: all systems factored together (FP32, one
    union pattern analysed once) and solved in batched launches (one CTA per
    system) with FP64 refinement to relres 1e-8.  A step = factor + solve of
    the whole batch; value = systems solved per second."""
    import torch

    import culip_b200 as cb

    world, rank, local = _dist()
    torch.cuda.set_device(local)
    block, tuning = 32, None
    if args.tune:
        block, tuning = tune_batch_block(args, local)
    syst = batch_systems(args.batch, block=block)
    rp, ci, v, bs, off = cb.union_systems(syst)
    N, nnz = len(rp) - 1, len(ci)
    b = np.concatenate([cb.normal_vector(cb.SEED + 4000 + 100000 + i, len(sy[0]) - 1) for i, sy in enumerate(syst)])
    stream = torch.cuda.current_stream()
    h = cb.Handle(local, stream)
    t0 = time.perf_counter()
    P = cb.Pattern(h, rp, ci, bs, 0, 1.0, cb.F32, system_row_offsets=off)
    analysis_s = time.perf_counter() - t0
    F = cb.Factor(P)
    B = cb.Batch(P, off)
    d_rp = torch.from_numpy(rp).cuda()
    d_ci = torch.from_numpy(ci).cuda()
    d_v = torch.from_numpy(v).cuda()
    d_v32 = d_v.float()
    d_b = torch.from_numpy(b).cuda()
    d_x = torch.zeros(N, dtype=torch.float64, device="cuda")
    A = cb.CsrOperator(h, d_rp, d_ci, d_v)
    flush = L2Flush()
    tol, inner_tol, inner_it, max_ref = 1e-8, 1e-6, args.max_it, args.max_refine
    stats = {}

    def step():
        F.compute_graph(d_v32, cb.PIV_BK, 0.0)
        rel, its, steps, st = cb.batch_sqmr_refine(B, A, F, d_b, d_x, tol, inner_tol, inner_it, max_ref)
        stats.update(rel=rel, its=its, steps=steps, st=st)

    for _ in range(args.warmup):
        flush.fill_(1.0)
        step()
    torch.cuda.synchronize()
    h.launch_count(reset=True)
    clocks = ClockSampler(local)
    clocks.start()
    ms = []
    for i in range(args.steps):
        flush.fill_(float(i))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        step()
        e1.record(stream)
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    ck = clocks.stop()
    launches = h.launch_count(reset=True)
    total_ms = float(np.sum(ms))
    fac_ms, _ = F.stats()
    conv = float(np.mean(stats["st"] == 0))
    # e2e: FP64 values and b from pinned host memory, FP32 cast on the device, x back
    hv = torch.from_numpy(v).pin_memory()
    hb = torch.from_numpy(b).pin_memory()
    hx = torch.empty(N, dtype=torch.float64).pin_memory()
    e_ms = []
    for i in range(max(2, min(args.steps, 3))):
        flush.fill_(float(i))
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        d_v.copy_(hv, non_blocking=True)
        d_b.copy_(hb, non_blocking=True)
        d_v32.copy_(d_v)
        step()
        hx.copy_(d_x, non_blocking=True)
        e1.record(stream)
        torch.cuda.synchronize()
        e_ms.append(e0.elapsed_time(e1))
    # the factorization and one batched solve of every system as ONE graph
    # launch (culipx_batch_factor_solve_graph): first call captures, then timed replays
    xg = torch.zeros_like(d_x)
    cb.batch_factor_solve_graph(B, A, F, d_v32, d_b, xg, inner_tol, inner_it)
    g_ms, g_st = [], None
    for i in range(3):
        flush.fill_(float(i))
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        _, g_its, g_st = cb.batch_factor_solve_graph(B, A, F, d_v32, d_b, xg, inner_tol, inner_it)
        e1.record(stream)
        torch.cuda.synchronize()
        g_ms.append(e0.elapsed_time(e1))
    num = len(syst)
    single_graph = {"what": "factor + one batched SQMR solve of all systems (tol 1e-6, no refinement) as one CUDA "
                            "graph launch", "ms": float(np.mean(g_ms)),
                    "systems_per_s": num / (float(np.mean(g_ms)) / 1e3),
                    "quasi_residual_converged_fraction": float(np.mean(g_st == 0)),
                    "median_iterations": int(np.median(g_its))}
    out = {
        "metric": "KKT solves/s (batched uneven instances, FP32 factor + FP64 refinement to relres 1e-8)",
        "value": num * args.steps / (total_ms / 1e3), "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 factor / f64 refinement", "data": "synthetic (seeded KKT generator)",
        "config": {"workload": f"{num} KKT systems, n U[500,20000], m=n/2, A 4-8/col (band_half=32), "
                               f"H log-U[1e-4,1e4], blocks {block} "
                               f"({'culipx_tune_kkt_block on 4 sample systems' if tuning else 'fixed'}), BK, fill 0; "
                               f"union N={N} nnz={nnz}",
                   "block_tuning": tuning,
                   "solver": f"batched SQMR (one CTA per system), inner tol {inner_tol:g} max_it {inner_it}, "
                             f"FP64 refinement to {tol:g}, at most {max_ref} corrections",
                   "l2": L2Flush.NOTE,
                   "parallelism": "one GPU, systems as CTAs"},
        "converged_fraction": conv,
        "median_iterations": int(np.median(stats["its"])), "max_iterations": int(np.max(stats["its"])),
        "median_corrections": int(np.median(stats["steps"])),
        "max_true_relres_converged": float(np.max(stats["rel"][stats["st"] == 0])) if conv > 0 else None,
        "factor_ms": fac_ms, "analysis_s_once": analysis_s, "gpu_launches": int(launches), "clocks": ck,
        "e2e": {"value": num * len(e_ms) / (float(np.sum(e_ms)) / 1e3), "unit": "solves/s",
                "h2d_bytes_per_step": int(nnz * 8 + N * 8), "d2h_bytes_per_step": int(N * 8)},
        "single_graph": single_graph,
    }
    if rank == 0:
        print(json.dumps(out), flush=True)


def served_workload(num_patterns, seed_base):
    """Config 5: num_patterns KKT patterns, pattern j from sub-seed
    seed_base + j, n log-uniform in [1e3, 5e5], m = n // 2, A with 6 nonzeros
    per column (half in a band of half-width 32), initial H log-uniform in
    [1e-6, 1e6], delta = gamma = 1e-8, 32-row blocks."""
    import culip_b200 as cb

    rng = np.random.default_rng(seed_base)
    pats = []
    for j in range(num_patterns):
        n = int(round(10 ** rng.uniform(3, np.log10(5e5))))
        m = n // 2
        rp, ci, v = cb.kkt_generate(n, m, 6, 32, 1e-6, 1e6, seed=seed_base + j)
        pats.append((rp, ci, v, cb.kkt_blocking(n, m, 32), n))
    return pats


def run_served(args):
    """Served IPM stream: Poisson arrivals at --rate over the patterns for
    --duration seconds; request = the pattern's next IPM iteration (H times
    10^U(-1, 1), clipped to [1e-8, 1e8]) with 1-8 N(0,1) right-hand sides,
    submitted to the server when its arrival time has passed (host wall
    clock), solved to SQMR tol 1e-8.  value = requests completed / (time from
    the first arrival to the last completion); latency = submit to completion."""
    import culip_b200 as cb

    import torch

    world, rank, local = _dist()
    torch.cuda.set_device(local)
    seed_base = cb.SEED + 5000
    pats = served_workload(args.patterns, seed_base)
    rng = np.random.default_rng(seed_base + 999)
    # arrival trace
    t, arrivals = 0.0, []
    while True:
        t += rng.exponential(1.0 / args.rate)
        if t > args.duration:
            break
        arrivals.append((t, int(rng.integers(0, len(pats))), int(rng.integers(1, 9))))
    # per-pattern IPM state: the diagonal of H evolves request by request
    state = []
    for rp, ci, v, bs, n in pats:
        rows = np.repeat(np.arange(len(rp) - 1), np.diff(rp))
        d = np.nonzero((rows == ci) & (rows < n))[0]
        state.append([v.copy(), d])

    def make_request(j, nrhs):
        v, d = state[j]
        h = np.clip((v[d] - 1e-8) * 10.0 ** rng.uniform(-1, 1, len(d)), 1e-8, 1e8)
        v = v.copy()
        v[d] = h + 1e-8
        state[j][0] = v
        return v, rng.standard_normal((len(pats[j][0]) - 1, nrhs))

    if args.plain:
        return run_served_plain(args, pats, arrivals, make_request, local)
    srv = cb.Server(local, 0, 3, 512, 1e-8, args.max_it)
    srv.set_large_rows(args.large_rows)
    srv.set_refine(args.refine, 1e-6)
    t0 = time.perf_counter()
    prec = cb.F32 if args.precision == "f32" else cb.F64
    pids = [srv.add_pattern(rp, ci, bs, prec) for rp, ci, v, bs, n in pats]
    analysis_s = time.perf_counter() - t0
    # warm-up: one request per pattern (factor pools, workspaces)
    for j in range(len(pats)):
        srv.submit(pids[j], pats[j][2], np.zeros(len(pats[j][0]) - 1) + 1.0)
    while srv.stats()["done"] < len(pats):
        srv.progress(wait=True)
    clocks = ClockSampler(local)
    clocks.start()
    launches0 = srv.launch_count()
    ids = []
    start = time.perf_counter()
    k = 0
    reqs = arrivals
    while k < len(reqs) or srv.stats()["done"] < len(pats) + len(reqs):
        now = time.perf_counter() - start
        while k < len(reqs) and reqs[k][0] <= now:
            v, b = make_request(reqs[k][1], reqs[k][2])  # the request's values are built as it arrives
            ids.append(srv.submit(pids[reqs[k][1]], v, b))
            k += 1
        if srv.progress(wait=False) == 0 and k < len(reqs):
            time.sleep(min(0.0005, max(0.0, reqs[k][0] - (time.perf_counter() - start))))
        elif k >= len(reqs):
            srv.progress(wait=True)
    elapsed = time.perf_counter() - start
    ck = clocks.stop()
    launches = srv.launch_count() - launches0
    lat, its, conv, nrhs_tot = [], [], 0, 0
    for i in ids:
        x, it, st, l = srv.result(i)
        lat.append(l)
        its.extend(it.tolist())
        conv += int(np.sum(st == 0))
        nrhs_tot += len(st)
    lat = np.array(lat)
    out = {
        "metric": "KKT solves/s and p50/p99 latency (served IPM stream, "
                  + ("FP32 factor + FP64 SQMR" if args.precision == "f32" else "FP64 plain method") + " per request)",
        "value": len(ids) / elapsed, "unit": "requests/s", "n_gpus": world, "steps": len(ids), "warmup": len(pats),
        "ms_per_step": 1e3 * elapsed / max(len(ids), 1), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 factor / f64 recurrence" if args.precision == "f32" else "f64",
        "data": "synthetic (seeded KKT generator, Poisson arrivals)",
        "config": {"workload": f"{len(pats)} patterns, n log-U[1e3,5e5], m=n/2, A 6/col (band_half=32), "
                               f"Poisson {args.rate:g} req/s for {args.duration:g} s ({len(ids)} requests), "
                               f"1-8 RHS, H *= 10^U(-1,1) clipped [1e-8,1e8] per request",
                   "solver": f"server: 3 slots; patterns with N < {args.large_rows}: batched SQMR, one CTA per right-hand "
                             f"side; larger: the whole-GPU solver, right-hand sides in groups of up to 4, in "
                             f"exclusive batches; tol 1e-8, max_it {args.max_it}; FP64 refinement: "
                             f"{args.refine} corrections at most (inner tol 1e-6)", "parallelism": "one GPU"},
        "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                       "mean": float(lat.mean()), "max": float(lat.max())},
        "right_hand_sides": nrhs_tot, "converged_fraction": conv / max(nrhs_tot, 1),
        "median_iterations": int(np.median(its)) if its else None, "pattern_analysis_s_once": analysis_s,
        "clocks": ck, "gpu_launches": int(launches),
    }
    if rank == 0:
        print(json.dumps(out), flush=True)


def schur_update_stats(P, F, bs):
    """Sparsity of the block Schur updates of a computed factor, from its
    export: for every pivot block row k and every pair of its off-diagonal
    blocks (k, i), (k, j), i <= j, whose target block (i, j) exists in the
    pattern (level-based fill drops the rest), the update U_ki' D_k U_kj.
    F_alg counts 2 flops per product of a nonzero of U_ki and a nonzero of
    U_kj in the same row of block row k (1x1 pivots; the sparse work the
    update needs), F_tile 2 h_k h_i h_j (the dense tile product a tensor-core
    MMA would issue).  Returns the totals and histograms of nonzeros per
    off-diagonal block and of F_alg / F_tile per update."""
    pe = P.export()
    E = F.export()
    bs = np.asarray(bs, np.int64)
    off, col = pe["coarse_off"].astype(np.int64), pe["coarse_col"].astype(np.int64)
    cm = len(off) - 1
    rows = np.repeat(np.arange(cm), np.diff(off))
    exists = set(zip(rows.tolist(), col.tolist()))
    bo = E["blk_off"]
    nnz_blk, dens = [], []
    f_alg = f_tile = 0.0
    n_upd = 0
    for k in range(cm):
        hk = int(bs[k + 1] - bs[k])
        qs = [q for q in range(off[k], off[k + 1]) if col[q] > k]
        if not qs:
            continue
        rn = {}
        for q in qs:
            J = int(col[q])
            w = int(bs[J + 1] - bs[J])
            s0, s1 = int(bo[q]), int(bo[q + 1])
            idx, val = E["idx"][s0:s1], E["val"][s0:s1]
            keep = val != 0
            r = np.bincount(idx[keep] // w, minlength=hk)[:hk].astype(np.float64)
            rn[J] = r
            nnz_blk.append(int(keep.sum()))
        cols = sorted(rn)
        for a, i in enumerate(cols):
            for j in cols[a:]:
                if (i, j) not in exists:
                    continue
                fa = 2.0 * float(rn[i] @ rn[j])
                ft = 2.0 * hk * float(bs[i + 1] - bs[i]) * float(bs[j + 1] - bs[j])
                f_alg += fa
                f_tile += ft
                dens.append(fa / ft)
                n_upd += 1
    nnz_blk = np.array(nnz_blk)
    dens = np.array(dens) if dens else np.zeros(1)
    hist_edges = [0, 1, 2, 4, 8, 16, 32, 64, 128, 256, 512, 1025]
    h_nnz, _ = np.histogram(nnz_blk, bins=hist_edges)
    d_edges = [0, 1e-3, 3e-3, 1e-2, 3e-2, 0.1, 0.3, 1.0001]
    h_den, _ = np.histogram(dens, bins=d_edges)
    return {"updates": n_upd, "F_alg": f_alg, "F_tile": f_tile, "F_alg_over_F_tile": f_alg / max(f_tile, 1.0),
            "offdiag_blocks": int(len(nnz_blk)),
            "nnz_per_offdiag_block": {"median": float(np.median(nnz_blk)) if len(nnz_blk) else 0.0,
                                      "max": int(nnz_blk.max()) if len(nnz_blk) else 0,
                                      "histogram": {f"[{a},{b})": int(c) for a, b, c in
                                                    zip(hist_edges[:-1], hist_edges[1:], h_nnz)}},
            "update_density": {"median": float(np.median(dens)), "max": float(dens.max()),
                               "updates_at_least_0.1": int((dens >= 0.1).sum()),
                               "histogram": {f"[{a:g},{b:g})": int(c) for a, b, c in
                                             zip(d_edges[:-1], d_edges[1:], h_den)}}}


def run_schur(args):
    """The tensor-core question for the factorization: F_alg vs F_tile of the
    block Schur updates (schur_update_stats) of the FP32 factor of the
    mixed-precision workload (n = 1e6, m = 5e5) and of the FP64 factor of the
    scale workload, on their BK factors as the GPU computes them."""
    import torch

    import culip_b200 as cb

    torch.cuda.set_device(0)
    h = cb.Handle(0)
    res = {}
    for name, prec in (("mixed", cb.F32), ("scale", cb.F64)):
        cfg, rp, ci, v, bs, _ = _workload(name)
        P = cb.Pattern(h, rp, ci, bs, 0, 1.0, prec)
        F = cb.Factor(P)
        F.compute(torch.from_numpy(v).to(torch.float32 if prec == cb.F32 else torch.float64).cuda(), None,
                  cb.PIV_BK, 0.0)
        t0 = time.perf_counter()
        st = schur_update_stats(P, F, bs)
        st["analysis_s"] = time.perf_counter() - t0
        st["workload"] = _config_dict(name, cfg, len(ci))["workload"]
        res[name] = st
    print(json.dumps({"metric": "block Schur updates: F_alg / F_tile (tensor-core candidate work)", "configs": res}),
          flush=True)


def run_served_plain(args, pats, arrivals, make_request, local):
    """The served trace's requests through the plain FP64 single-solve path,
    back to back (throughput; arrival times ignored): per request the FP64
    factor of its values (each pattern analysed once, before the timing) and
    one culipx_sqmr_solve per right-hand side on the whole GPU.  value =
    requests / the device time of the whole run; the ratio of the served
    line's value to this one is the serving path's gain at the same iteration
    cap."""
    import torch

    import culip_b200 as cb

    h = cb.Handle(local)
    stream = torch.cuda.current_stream()
    fac = []
    for rp, ci, v, bs, n in pats:
        P = cb.Pattern(h, rp, ci, bs, 0, 1.0, cb.F64)
        F = cb.Factor(P)
        d_rp, d_ci = torch.from_numpy(rp).cuda(), torch.from_numpy(ci).cuda()
        d_v = torch.from_numpy(v).cuda()
        fac.append((P, F, cb.CsrOperator(h, d_rp, d_ci, d_v), d_v))
    # warm-up: one solve per pattern
    for (P, F, A, d_v), (rp, ci, v, bs, n) in zip(fac, pats):
        F.compute(d_v)
        x = torch.zeros(len(rp) - 1, dtype=torch.float64, device="cuda")
        cb.sqmr_solve(h, A, F, torch.ones_like(x), x, 1e-8, args.max_it)
    reqs = [make_request(j, nrhs) for _, j, nrhs in arrivals]
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    nrhs_tot, conv, its = 0, 0, []
    for (_, j, nrhs), (v, B) in zip(arrivals, reqs):
        P, F, A, d_v = fac[j]
        d_v.copy_(torch.from_numpy(v))
        F.compute(d_v)
        for c in range(B.shape[1]):
            b = torch.from_numpy(np.ascontiguousarray(B[:, c])).cuda()
            x = torch.zeros_like(b)
            res, it, st = cb.sqmr_solve(h, A, F, b, x, 1e-8, args.max_it)
            its.append(it)
            conv += int(st == 0)
            nrhs_tot += 1
    e1.record(stream)
    torch.cuda.synchronize()
    ck = clocks.stop()
    sec = e0.elapsed_time(e1) / 1e3
    out = {"metric": "KKT solves/s (served IPM stream's requests through the plain FP64 single-solve path)",
           "value": len(reqs) / sec, "unit": "requests/s", "n_gpus": 1, "steps": len(reqs), "warmup": len(pats),
           "ms_per_step": 1e3 * sec / max(len(reqs), 1), "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded KKT generator, the served trace's requests)",
           "config": {"workload": f"{len(pats)} patterns, {len(reqs)} requests, {nrhs_tot} right-hand sides "
                                  f"(the trace of --config served --rate {args.rate:g} --duration {args.duration:g})",
                      "solver": f"FP64 factor per request, culipx_sqmr_solve per right-hand side, tol 1e-8, max_it "
                                f"{args.max_it}", "parallelism": "one GPU, one solve at a time"},
           "right_hand_sides": nrhs_tot, "rhs_per_s": nrhs_tot / sec, "converged_fraction": conv / max(nrhs_tot, 1),
           "median_iterations": int(np.median(its)) if its else None, "clocks": ck}
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    a = _parse()
    if a.impl == "reference":
        run_reference(a)
    elif a.config == "schur":
        run_schur(a)
    elif a.config == "mixed":
        run_mixed(a)
    elif a.config == "spmv":
        run_spmv(a)
    elif a.config == "batch":
        run_batch(a)
    elif a.config == "served":
        run_served(a)
    else:
        run_culipx(a)
