"""ISDF solves/s on B200 (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--config si64|si8|si216] [--precision fp64|mixed]

A step is one full ISDF solve (weight -> K-means selection -> Z C^T GEMM with
the Hadamard epilogue -> C C^T -> Cholesky -> triangular solves) through the
public API, check = false, on synthetic Kohn-Sham-like orbitals of the
configured shape (libisdf_b200/synth.py, seeded). Default workload: the
Si64-like shape (80^3 grid, 256 states, S1 = S2 = all states, mu = 2048,
100 K-means iterations, plain FP64).

value: solves/s with psi resident in HBM (device time, CUDA events on the
solve stream; max over ranks). e2e: the same through the public API from
host buffers, with the H2D copy of psi and the D2H copy of theta inside the
timed region. Under torchrun each rank runs independent solves on its own GPU
(the path does not shard: replicas only, weak scaling, no collective on the
data path).

--impl reference times the reference's own CPU implementation
(oracle/_ref: the reference sources compiled with single-rank shims) on a
bounded sample of the same workload and extrapolates to solves/s.
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

METRIC = "ISDF solves/s"


def _rank_env():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                      "--format=csv,noheader,nounits"], capture_output=True,
                                     text=True, timeout=5).stdout.strip()
                if out:
                    self.rows.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4)
                          if len(r) > 5 + i and r[5 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


def _measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f), "MEASURED_PEAKS.json"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def _fp64_peak_tflops(torch):
    """cuBLAS DGEMM 8192^3 (best of 5) on this GPU: the FP64 denominator."""
    a = torch.randn(8192, 8192, dtype=torch.float64, device="cuda")
    b = torch.randn_like(a)
    for _ in range(2):
        a @ b
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        a @ b
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    torch.cuda.empty_cache()
    return 2 * 8192 ** 3 / (best * 1e-3) / 1e12


def max_over_ranks(x: float, dist=None, device="cpu") -> float:
    """The slowest rank's figure: every rank calls this at the same point."""
    if dist is None:
        return float(x)
    import torch

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(world: int, steps: int, t_ms: float) -> float:
    """Whole-job solves/s: every rank ran `steps` independent solves; t_ms is
    the max over ranks of the timed region."""
    return world * steps / (t_ms * 1e-3)


# ------------------------------------------------------------------ reference arm
def reference_sample(shape, iters: int, repeats: int = 1):
    """Seconds per solve of the reference's CPU path, from a bounded sample:
    one K-means Lloyd step of the reference (its pdist2 + findMin over all
    grid points, utility.cpp:878-901) timed at full size, times the iteration
    count, plus the reference's getbasis_MPI fit on a 1/16 row block of the
    grid (its cost is linear in the rows), times 16."""
    from oracle import ref
    from libisdf_b200 import synth

    psi = synth.shape_orbitals(shape, 1)
    t_iter = ref.bench_kmeans_step(psi.shape[0], shape.mu, repeats)
    t_fit = ref.bench_getbasis_rows(psi, shape, 16, repeats)
    return iters * t_iter + 16 * t_fit, {
        "kind": "reference", "cores": os.cpu_count(),
        "sample": (f"{shape.name}: one reference K-means step (pdist2+findMin over {shape.ng} "
                   f"points x {shape.mu} centroids) x {iters} iterations + reference getbasis_MPI "
                   f"on {shape.ng // 16} rows x 16; OpenBLAS threads = {os.cpu_count()}, "
                   "K-means single-threaded as in the reference")}


def run_reference(args, shape):
    rank, world, _ = _rank_env()
    if rank != 0:
        return
    from oracle import ref

    if not ref.available():
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref/libisdf_ref.so not built (needs the reference checkout)"}))
        return
    for _ in range(args.warmup):
        reference_sample(shape, shape.kmeans_iters)
    times = []
    info = None
    for _ in range(args.steps):
        t, info = reference_sample(shape, shape.kmeans_iters)
        times.append(t)
    t = float(np.mean(times))
    v = 1.0 / t
    line = {"metric": METRIC, "value": v, "unit": "solves/s", "impl": "reference",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": shape.name, "ng": shape.ng, "nstate": shape.nstate,
                       "mu": shape.mu, "kmeans_iters": shape.kmeans_iters,
                       "selector": "Kmeans", "precision": "fp64"},
            "cpu_baseline": dict(info, value=v, unit="solves/s"),
            "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def _int8_peak_tops(torch):
    """cuBLASLt INT8 GEMM (torch._int_mm, 8192^3, best of 5): the INT8
    tensor-core denominator for the mixed form's GEMMs."""
    try:
        a = torch.randint(-127, 128, (8192, 8192), dtype=torch.int8, device="cuda")
        b = torch.randint(-127, 128, (8192, 8192), dtype=torch.int8, device="cuda").t()
        for _ in range(2):
            torch._int_mm(a, b)
        torch.cuda.synchronize()
        best = 1e30
        for _ in range(5):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            torch._int_mm(a, b)
            e1.record()
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1))
        del a, b
        torch.cuda.empty_cache()
        return 2 * 8192 ** 3 / (best * 1e-3) / 1e12, "cuBLASLt INT8 GEMM 8192^3 measured in this run"
    except Exception as e:  # noqa: BLE001
        peaks, _ = _measured_peaks()
        return 2.0 * peaks["bf16_tflops"], f"2 x measured dense BF16 (INT8 GEMM unavailable: {e})"


def mixed_vs_fp64(torch, shape, psi, d_theta, piv, rk, solve_fp64, n_rows=2048, n_pairs=1024,
                  seed=0):
    """Accuracy of the mixed-precision result in d_theta against the FP64
    form on the same inputs: relative Frobenius error of the fitted pair
    densities theta C (and of theta) on sampled grid rows and pairs. Runs one
    FP64 solve into d_theta (outside any timed region)."""
    rng = np.random.default_rng(seed)
    ng = psi.shape[0]
    rows = np.sort(rng.choice(ng, size=min(n_rows, ng), replace=False))
    idx = torch.from_numpy(rows).cuda()
    th_m = d_theta[:rk].index_select(1, idx).T.cpu().numpy()
    piv_m = piv[:rk].copy()
    solve_fp64()
    th_f = d_theta[:rk].index_select(1, idx).T.cpu().numpy()
    if not np.array_equal(piv_m, piv[:rk]):
        return {"error": "piv differs between the forms"}
    lo1, lo2 = shape.nocc - shape.nv1, shape.nocc - shape.nv2
    i = lo1 + rng.integers(0, shape.nv1 + shape.nc1, size=n_pairs)
    j = lo2 + rng.integers(0, shape.nv2 + shape.nc2, size=n_pairs)
    pm = psi[piv_m]  # rk x nstate
    C = pm[:, i] * pm[:, j]
    fd_m, fd_f = th_m @ C, th_f @ C
    return {"fitted_densities_rel": float(np.linalg.norm(fd_m - fd_f) / np.linalg.norm(fd_f)),
            "theta_rel": float(np.linalg.norm(th_m - th_f) / np.linalg.norm(th_f)),
            "rows": int(len(rows)), "pairs": int(n_pairs),
            "against": "the FP64 form on the same inputs (parity-tested against the oracle)"}


# ------------------------------------------------------------------ our arm
def run_ours(args, shape):
    import torch

    import libisdf_b200 as isdf
    from libisdf_b200 import synth

    rank, world, local = _rank_env()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    psi = synth.shape_orbitals(shape, 1, device="cuda")
    ng, mu = shape.ng, shape.mu
    h_psi = torch.from_numpy(np.ascontiguousarray(psi.T)).pin_memory()
    d_psi = h_psi.cuda()
    d_theta = torch.empty((mu, ng), dtype=torch.float64, device="cuda")
    piv = np.zeros(ng, dtype=np.int32)
    dom = isdf.Domain(length=(shape.length,) * 3, num_grid=(shape.n,) * 3)
    stream = torch.cuda.Stream()
    prec = isdf.PRECISION_MIXED if args.precision == "mixed" else isdf.PRECISION_FP64
    opts = isdf.Options(stream=stream.cuda_stream, precision=prec,
                        qrcp_oversample=args.qrcp_factor, qrcp_seed=args.qrcp_seed,
                        mixed_slices=args.mixed_slices)
    s1 = "QRCP" if args.selector == "qrcp" else "Kmeans"

    def solve(theta=None, psi_d=None):
        return isdf.ISDF(d_psi if psi_d is None else psi_d, dom, shape.nocc, shape.nstate,
                         shape.nv1, shape.nc1, shape.nv2, shape.nc2, mu,
                         d_theta if theta is None else theta, piv, shape.kmeans_iters, s1=s1,
                         options=opts)

    fp64_peak = _fp64_peak_tflops(torch)
    int8_peak = _int8_peak_tops(torch) if args.precision == "mixed" else None
    with torch.cuda.stream(stream):
        for _ in range(max(3, args.warmup)):
            rep = solve()
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        lat = []
        stage = []
        launches = []
        with ClockSampler(local) as clk:
            e_start = torch.cuda.Event(enable_timing=True)
            e_end = torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e_start.record(stream)
            for _ in range(args.steps):
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                rep = solve()
                e1.record(stream)
                e1.synchronize()
                lat.append(e0.elapsed_time(e1))
                stage.append((rep.t_select_ms, rep.t_fit_ms, rep.t_solve_ms, rep.t_zct_ms,
                              rep.t_chol_ms, rep.t_gemm_ms))
                launches.append(rep.kernel_launches)
            e_end.record(stream)
            torch.cuda.synchronize()
        t_ms = max_over_ranks(e_start.elapsed_time(e_end), dist, "cuda")
        if dist:
            dist.barrier()

        # End to end from host buffers, as a caller that consumes theta on the
        # host runs it: every step copies its psi in (pinned host -> HBM),
        # solves, and copies theta out (HBM -> pinned host), in a steady
        # pipeline: the psi of step i+1 is copied in on an H2D stream and the
        # theta of step i copied out on a D2H stream while step i+1 solves
        # (two device psi and theta buffers when HBM allows, else one of each
        # and those copies do not overlap). At least 8 steps, so that the
        # pipeline's fill and drain are a small part of the timed region.
        h_theta = torch.empty((mu, ng), dtype=torch.float64).pin_memory()
        e2e_steps = max(8, args.steps)
        free_b, _ = torch.cuda.mem_get_info()
        thetas = [d_theta]
        if free_b > d_theta.numel() * 8 + (8 << 30):
            thetas.append(torch.empty_like(d_theta))
            free_b -= d_theta.numel() * 8
        psis = [d_psi]
        if free_b > d_psi.numel() * 8 + (8 << 30):
            psis.append(torch.empty_like(d_psi))
        copy_stream = torch.cuda.Stream()
        h2d_stream = torch.cuda.Stream()
        done = [None] * len(thetas)      # theta buffer copied out
        used = [None] * len(psis)        # psi buffer no longer read by a solve
        ready = [None] * len(psis)       # psi buffer holds its step's input

        def fetch(k):
            b = k % len(psis)
            if used[b] is not None:
                h2d_stream.wait_event(used[b])
            with torch.cuda.stream(h2d_stream):
                psis[b].copy_(h_psi, non_blocking=True)
            ready[b] = torch.cuda.Event()
            ready[b].record(h2d_stream)

        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        h2d_stream.wait_event(e0)
        fetch(0)
        for i in range(e2e_steps):
            pb, tb = i % len(psis), i % len(thetas)
            stream.wait_event(ready[pb])
            if done[tb] is not None:
                stream.wait_event(done[tb])
            if len(psis) > 1 and i + 1 < e2e_steps:
                fetch(i + 1)  # into the other buffer, beside this solve
            rep = solve(thetas[tb], psis[pb])
            solved = torch.cuda.Event()
            solved.record(stream)
            used[pb] = solved
            if len(psis) == 1 and i + 1 < e2e_steps:
                fetch(i + 1)
            copy_stream.wait_event(solved)
            with torch.cuda.stream(copy_stream):
                # in 256 MB pieces, so that the library's small state reads
                # of the next solve are not queued behind one long copy
                src, dst = thetas[tb].view(-1), h_theta.view(-1)
                piece = 1 << 25
                for o in range(0, src.numel(), piece):
                    dst[o:o + piece].copy_(src[o:o + piece], non_blocking=True)
            done[tb] = torch.cuda.Event()
            done[tb].record(copy_stream)
        stream.wait_stream(copy_stream)
        e1.record(stream)
        torch.cuda.synchronize()
        e2e_ms = max_over_ranks(e0.elapsed_time(e1), dist, "cuda")
        e2e_bufs = len(thetas)
        e2e_psi_bufs = len(psis)
        del thetas, psis

    if dist:
        dist.destroy_process_group()
    if rank != 0:
        return
    accuracy = None
    if args.precision == "mixed":
        opts64 = isdf.Options(stream=stream.cuda_stream, precision=isdf.PRECISION_FP64,
                              qrcp_oversample=args.qrcp_factor, qrcp_seed=args.qrcp_seed)

        def solve_fp64():
            with torch.cuda.stream(stream):
                isdf.ISDF(d_psi, dom, shape.nocc, shape.nstate, shape.nv1, shape.nc1, shape.nv2,
                          shape.nc2, mu, d_theta, piv, shape.kmeans_iters, s1=s1, options=opts64)
            torch.cuda.synchronize()

        accuracy = mixed_vs_fp64(torch, shape, psi, d_theta, piv, rep.rk_eff, solve_fp64)
    peaks, peak_src = _measured_peaks()
    v = replica_value(world, args.steps, t_ms)
    rk = rep.rk_eff
    t_solve_ms = float(np.median([s[2] for s in stage]))
    t_gemm_ms = float(np.median([s[5] for s in stage]))
    if args.precision == "mixed":
        # Dominant kernel: k_ozaki_gemm, the two triangular products
        # Y = Z L^-T and theta = Y L^-1 as INT8 digit-pair GEMMs; issued INT8
        # ops per solve: 2 GEMMs x 2 x Ng x rk x (rk/2 + 32) x S(S+1)/2 (each
        # tile runs the K range its triangular factor leaves nonzero). Time:
        # CUDA events around the two launches on the solve stream.
        S = args.mixed_slices
        ops = 2 * 2.0 * ng * rk * (rk / 2 + 32) * S * (S + 1) / 2
        achieved = ops / (t_gemm_ms * 1e-3) / 1e12 if t_gemm_ms > 0 else None
        roofline = {"kernel": "k_ozaki_gemm (Y = Z L^-T and theta = Y L^-1, INT8 digit pairs)",
                    "bound": "tensor", "achieved": achieved, "peak": int8_peak[0],
                    "unit": "TOPS (INT8)", "frac": (achieved / int8_peak[0]) if achieved else None,
                    "peak_source": int8_peak[1],
                    "emulated_fp64_tflops": (2.0 * 2 * ng * rk * (rk / 2 + 32) /
                                             (t_gemm_ms * 1e-3) / 1e12) if t_gemm_ms > 0 else None,
                    "traffic": None}
    else:
        # Dominant kernel: k_trsm_ws, the two triangular sweeps as in-place
        # FP64 tensor-core GEMMs (warp-specialised bulk-copy tile). Algorithmic flops per solve: 2*Ng*rk^2
        # (Ng*rk^2 per sweep). Its time is the triangular-solve stage on the
        # solve stream (CUDA events in the library around the stage: the
        # k_trsm_ws launches plus the small k_build_w launches between
        # them), so the rate is a slight underestimate of the kernel's own.
        achieved = 2.0 * ng * rk * rk / (t_solve_ms * 1e-3) / 1e12 if t_solve_ms > 0 else None
        # DRAM traffic of one launch: 8.40 B per grid row and solved column
        # (dram__bytes_read.sum + dram__bytes_write.sum of ncu on the 40^3-grid
        # case), times the mean solved width of a launch over both sweeps
        # (rk/2 + 32 columns).
        roofline = {"kernel": "k_trsm_ws (both sweeps of the triangular solve)",
                    "bound": "tensor", "achieved": achieved, "peak": fp64_peak,
                    "unit": "TFLOP/s", "frac": (achieved / fp64_peak) if achieved else None,
                    "peak_source": ("cuBLAS DGEMM 8192^3 measured in this run: the FP64 "
                                    "denominator (the measured-peaks file holds HBM and BF16 "
                                    f"figures only; HBM {peaks.get('hbm_gbs')} GB/s from "
                                    f"{peak_src})"),
                    "traffic": 8.40 * ng * (rk / 2 + 32),
                    "traffic_note": "bytes per launch (mean over the sweep), scaled from the "
                                    "ncu capture at Ng = 64000 by rows x solved columns"}
    line = {
        "metric": METRIC, "value": v, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": max(3, args.warmup), "ms_per_step": t_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": shape.name, "ng": ng, "nstate": shape.nstate, "mu": mu,
                   "rk_eff": rk, "kmeans_iters": rep.kmeans_iters, "npt": rep.npt,
                   "kmeans_search_frac": round(float(rep.kmeans_search_frac), 4), "selector": s1,
                   **({"qrcp_oversample": args.qrcp_factor, "qrcp_seed": args.qrcp_seed}
                      if s1 == "QRCP" else {}),
                   "precision": args.precision,
                   **({"mixed_slices": args.mixed_slices} if args.precision == "mixed" else {}),
                   "parallelism": f"replicas x{world}",
                   "l2": (f"inputs larger than L2 (psi {ng * shape.nstate * 8 / 1e9:.2f} GB, "
                          f"theta {ng * mu * 8 / 1e9:.2f} GB; L2 126 MB)")},
        "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))},
        "stages_ms": {"select_wall": float(np.median([s[0] for s in stage])),
                      "fit_wall": float(np.median([s[1] for s in stage])),
                      "zct_gemm": float(np.median([s[3] for s in stage])),
                      "cct_cholesky": float(np.median([s[4] for s in stage])),
                      "triangular_solve": t_solve_ms,
                      "triangular_gemms": t_gemm_ms},
        "roofline": roofline,
        "e2e": {"value": replica_value(world, e2e_steps, e2e_ms), "unit": "solves/s",
                "h2d_bytes_per_step": int(h_psi.numel() * 8),
                "d2h_bytes_per_step": int(h_theta.numel() * 8 + piv.nbytes),
                "steps": e2e_steps, "theta_buffers": e2e_bufs, "psi_buffers": e2e_psi_bufs},
        "gpu_launches": int(sum(launches)),
        "mixed_vs_fp64": accuracy,
        "clocks": clk.summary(),
    }
    if world == 1 and not args.no_cpu_baseline and s1 == "QRCP":
        line["cpu_baseline"] = {"value": None, "unit": "solves/s",
                                "unavailable": "the reference's QRCP selector runs ScaLAPACK "
                                               "pdgeqpf, which cannot be built here"}
    elif world == 1 and not args.no_cpu_baseline:
        try:
            t_cpu, info = reference_sample(shape, rep.kmeans_iters)
            line["cpu_baseline"] = dict(info, value=1.0 / t_cpu, unit="solves/s")
        except Exception as e:  # the reference build is optional on the box
            line["cpu_baseline"] = {"value": None, "unit": "solves/s",
                                    "unavailable": str(e)[:200]}
    print(json.dumps(line), flush=True)


def run_select(args, shape):
    """--stage select: the K-means selection alone (weight computed once),
    selections/s; a small-footprint command for profiling the K-means kernels
    at full grid size (psi, the weight and the K-means workspace only)."""
    import torch

    import libisdf_b200 as isdf
    from libisdf_b200 import synth

    torch.cuda.set_device(0)
    psi = synth.shape_orbitals(shape, 1, device="cuda")
    d_psi = torch.from_numpy(np.ascontiguousarray(psi.T)).cuda()
    d_w = torch.empty(shape.ng, dtype=torch.float64, device="cuda")
    dom = isdf.Domain(length=(shape.length,) * 3, num_grid=(shape.n,) * 3)
    stream = torch.cuda.Stream()
    isdf.kmeans_weight(d_psi, shape.ng, shape.nstate, shape.nocc, shape.nv1, shape.nc1, shape.nv2,
                       shape.nc2, d_w, stream=stream.cuda_stream)
    torch.cuda.synchronize()
    for _ in range(max(3, args.warmup)):
        isdf.kmeans_select(dom, d_w, shape.mu, shape.kmeans_iters, stream=stream.cuda_stream)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        _, rk, iters, npt = isdf.kmeans_select(dom, d_w, shape.mu, shape.kmeans_iters,
                                               stream=stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize()
    t_ms = e0.elapsed_time(e1)
    print(json.dumps({"metric": "K-means selections/s", "value": args.steps / (t_ms * 1e-3),
                      "unit": "selections/s", "n_gpus": 1, "steps": args.steps,
                      "warmup": max(3, args.warmup), "ms_per_step": t_ms / args.steps,
                      "higher_is_better": True, "dtype": "f64", "data": "synthetic",
                      "config": {"workload": shape.name, "ng": shape.ng, "mu": shape.mu,
                                 "rk_eff": rk, "kmeans_iters": iters, "npt": npt}}), flush=True)


def run_serve(args):
    """--serve: the serving mix (60 % Si8-like, 30 % Si64-like, 10 % Si216-like
    requests, K-means, --precision) arriving as a Poisson process at --rate
    requests/s, through the continuous-batching server (isdf_server_*).
    Latency is arrival -> completion as the client sees it (it includes any
    wait for a free output buffer); throughput is requests / (last completion
    - first arrival). psi comes from a small pool per shape (seeds 100, 101,
    ...), the request index picking the seed; every in-flight request has its
    own theta and piv."""
    import threading

    import torch

    import libisdf_b200 as isdf
    from libisdf_b200 import synth

    torch.cuda.set_device(0)
    shapes = [synth.SI8, synth.SI64, synth.SI216]
    pool_seeds = [4, 2, 1]
    theta_bufs = [8, 4, 1]
    mix = [0.6, 0.3, 0.1]
    if args.serve_mix != "standard":
        # one shape only (the served form's throughput at that size)
        k1 = {"si8": 0, "si64": 1, "si216": 2}[args.serve_mix]
        mix = [1.0 if k == k1 else 0.0 for k in range(3)]
        pool_seeds = [1 if k == k1 else 0 for k in range(3)]
        theta_bufs = [args.slots if k == k1 else 0 for k in range(3)]
    rng = np.random.default_rng(args.serve_seed)
    n_req = args.requests
    kinds = rng.choice(3, size=n_req, p=mix)
    arrivals = np.cumsum(rng.exponential(1.0 / args.rate, size=n_req))
    prec = isdf.PRECISION_MIXED if args.precision == "mixed" else isdf.PRECISION_FP64
    opts = isdf.Options(precision=prec)
    psi = {k: [torch.from_numpy(np.ascontiguousarray(
        synth.shape_orbitals(shapes[k], 100 + j, device="cuda").T)).cuda()
        for j in range(pool_seeds[k])] for k in range(3)}
    free = {k: [torch.empty((shapes[k].mu, shapes[k].ng), dtype=torch.float64, device="cuda")
                for _ in range(theta_bufs[k])] for k in range(3)}
    doms = [isdf.Domain(length=(sh.length,) * 3, num_grid=(sh.n,) * 3) for sh in shapes]
    torch.cuda.synchronize()

    budget = 0
    if args.hbm_budget_gb > 0:
        budget = int(args.hbm_budget_gb * (1 << 30))
    elif args.hbm_budget_gb < 0:  # all that is free now, less 4 GiB
        budget = max(0, torch.cuda.mem_get_info()[0] - (4 << 30))
    srv = isdf.Server(slots=args.slots, hbm_budget_bytes=budget)
    lock = threading.Condition()
    inflight = {}  # ticket -> (kind, theta, arrival index)
    done_at = np.zeros(n_req)

    def submit(k, i, theta):
        sh = shapes[k]
        piv = np.zeros(sh.ng, dtype=np.int32)
        return srv.submit(psi[k][i % pool_seeds[k]], doms[k], sh.nocc, sh.nstate, sh.nv1, sh.nc1,
                          sh.nv2, sh.nc2, sh.mu, theta, piv, sh.kmeans_iters, options=opts)

    # warm-up: one request of each shape served (workspaces, graphs)
    for k in range(3):
        if pool_seeds[k]:
            st, _ = srv.wait(submit(k, 0, free[k][0]))
            assert st == 0, isdf.lib().isdf_last_error()

    stop = threading.Event()

    def poller():
        while not stop.is_set() or inflight:
            with lock:
                items = list(inflight.items())
            finished = []
            for t, (k, th, i) in items:
                state, st = srv.poll(t)
                if state == 2:
                    done_at[i] = time.perf_counter()
                    finished.append((t, k, th, st))
            if finished:
                with lock:
                    for t, k, th, st in finished:
                        srv.wait(t)
                        del inflight[t]
                        free[k].append(th)
                        if st != 0:
                            inflight_errors.append(t)
                    lock.notify_all()
            time.sleep(0.0005)

    inflight_errors = []
    th_poll = threading.Thread(target=poller, daemon=True)
    th_poll.start()
    t0 = time.perf_counter()
    arr_at = t0 + arrivals
    with ClockSampler(0) as clk:
        for i in range(n_req):
            k = int(kinds[i])
            dt = arr_at[i] - time.perf_counter()
            if dt > 0:
                time.sleep(dt)
            with lock:
                while not free[k]:
                    lock.wait()
                theta = free[k].pop()
                t = submit(k, i, theta)
                inflight[t] = (k, theta, i)
        stop.set()
        th_poll.join()
    stats = srv.stats()
    srv.close()
    lat = (done_at - arr_at) * 1e3
    span = done_at.max() - arr_at[0]
    line = {"metric": "served ISDF solves/s (serving mix)", "value": n_req / span,
            "unit": "solves/s", "n_gpus": 1, "higher_is_better": True, "dtype": "f64",
            "data": "synthetic", "precision": args.precision,
            "config": {"workload": ("serving mix: 60 % Si8-like, 30 % Si64-like, 10 % Si216-like, "
                                    "K-means" if args.serve_mix == "standard" else
                                    f"served {args.serve_mix} requests only, K-means"),
                       "requests": n_req, "rate_per_s": args.rate,
                       "hbm_budget_bytes": budget,
                       "slots": args.slots, "psi_pool_seeds": pool_seeds,
                       "theta_buffers": theta_bufs,
                       "mix_counts": [int((kinds == k).sum()) for k in range(3)]},
            "latency_ms": {"p50": float(np.percentile(lat, 50)),
                           "p99": float(np.percentile(lat, 99)),
                           "p50_by_shape": {shapes[k].name: float(np.percentile(lat[kinds == k], 50))
                                            for k in range(3) if (kinds == k).any()}},
            "errors": len(inflight_errors),
            "server": {k: stats[k] for k in stats if k in ("completed", "peak_concurrency",
                                                              "p50_ms", "p99_ms", "peak_bytes")},
            "clocks": clk.summary()}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", choices=["si8", "si64", "si216", "si64c"], default="si64")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64")
    ap.add_argument("--mixed-slices", type=int, choices=[5, 6, 7], default=6,
                    help="INT8 digits per operand in the mixed form (Options.mixed_slices)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--selector", choices=["kmeans", "qrcp"], default="kmeans")
    ap.add_argument("--qrcp-factor", type=float, default=1.5,
                    help="QRCP oversampling (numPre = round(sqrt(f mu)); the reference uses 1.5)")
    ap.add_argument("--qrcp-seed", type=int, default=41)
    ap.add_argument("--stage", choices=["solve", "select"], default="solve",
                    help="select: time the K-means selection alone (profiling aid)")
    ap.add_argument("--serve", action="store_true",
                    help="the serving mix through isdf_server_* (Poisson arrivals)")
    ap.add_argument("--requests", type=int, default=128)
    ap.add_argument("--rate", type=float, default=4.0, help="arrivals per second (--serve)")
    ap.add_argument("--slots", type=int, default=4)
    ap.add_argument("--serve-seed", type=int, default=7)
    ap.add_argument("--serve-mix", choices=["standard", "si8", "si64", "si216"], default="standard",
                    help="standard: 60/30/10 Si8/Si64/Si216; else one shape only")
    ap.add_argument("--hbm-budget-gb", type=float, default=0.0,
                    help="server workspace budget (0: the library default, -1: all free less 4 GiB)")
    args = ap.parse_args()
    from libisdf_b200 import synth

    shape = synth.SHAPES[args.config]
    if args.impl == "reference":
        run_reference(args, shape)
    elif args.serve:
        run_serve(args)
    elif args.stage == "select":
        run_select(args, shape)
    else:
        run_ours(args, shape)


if __name__ == "__main__":
    main()
