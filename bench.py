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
    opts = isdf.Options(stream=stream.cuda_stream, precision=prec)

    def solve():
        return isdf.ISDF(d_psi, dom, shape.nocc, shape.nstate, shape.nv1, shape.nc1, shape.nv2,
                         shape.nc2, mu, d_theta, piv, shape.kmeans_iters, options=opts)

    fp64_peak = _fp64_peak_tflops(torch)
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
                              rep.t_chol_ms))
                launches.append(rep.kernel_launches)
            e_end.record(stream)
            torch.cuda.synchronize()
        t_ms = max_over_ranks(e_start.elapsed_time(e_end), dist, "cuda")
        if dist:
            dist.barrier()

        # end to end from host buffers: H2D psi, solve, D2H theta
        h_theta = torch.empty((mu, ng), dtype=torch.float64).pin_memory()
        e2e_steps = max(1, min(args.steps, 3))
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(e2e_steps):
            d_psi.copy_(h_psi, non_blocking=True)
            rep = solve()
            h_theta.copy_(d_theta, non_blocking=True)
        e1.record(stream)
        torch.cuda.synchronize()
        e2e_ms = max_over_ranks(e0.elapsed_time(e1), dist, "cuda")

    if dist:
        dist.destroy_process_group()
    if rank != 0:
        return
    peaks, peak_src = _measured_peaks()
    v = replica_value(world, args.steps, t_ms)
    # Dominant kernel: k_trsm_gemm, the two triangular sweeps as in-place FP64
    # tensor-core GEMMs. Algorithmic flops per solve: 2*Ng*rk^2 (Ng*rk^2 per
    # sweep). Its time is the triangular-solve stage on the solve stream
    # (CUDA events in the library around the stage: the k_trsm_gemm launches
    # plus the small k_build_w launches between them), so the rate is a
    # slight underestimate of the kernel's own.
    rk = rep.rk_eff
    t_solve_ms = float(np.median([s[2] for s in stage]))
    achieved = 2.0 * ng * rk * rk / (t_solve_ms * 1e-3) / 1e12 if t_solve_ms > 0 else None
    # DRAM traffic of one launch: 8.37 B per grid row and solved column
    # (dram__bytes_read.sum + dram__bytes_write.sum of ncu on the 40^3-grid
    # case), times the mean solved width of a launch over both sweeps
    # (rk/2 + 32 columns).
    traffic = 8.37 * ng * (rk / 2 + 32)
    line = {
        "metric": METRIC, "value": v, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": max(3, args.warmup), "ms_per_step": t_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": shape.name, "ng": ng, "nstate": shape.nstate, "mu": mu,
                   "rk_eff": rk, "kmeans_iters": rep.kmeans_iters, "selector": "Kmeans",
                   "precision": args.precision, "parallelism": f"replicas x{world}",
                   "l2": (f"inputs larger than L2 (psi {ng * shape.nstate * 8 / 1e9:.2f} GB, "
                          f"theta {ng * mu * 8 / 1e9:.2f} GB; L2 126 MB)")},
        "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))},
        "stages_ms": {"select_wall": float(np.median([s[0] for s in stage])),
                      "fit_wall": float(np.median([s[1] for s in stage])),
                      "zct_gemm": float(np.median([s[3] for s in stage])),
                      "cct_cholesky": float(np.median([s[4] for s in stage])),
                      "triangular_solve": t_solve_ms},
        "roofline": {"kernel": "k_trsm_gemm (both sweeps of the triangular solve)",
                     "bound": "tensor", "achieved": achieved, "peak": fp64_peak,
                     "unit": "TFLOP/s", "frac": (achieved / fp64_peak) if achieved else None,
                     "peak_source": ("cuBLAS DGEMM 8192^3 measured in this run: the FP64 "
                                     "denominator (the measured-peaks file holds HBM and BF16 "
                                     f"figures only; HBM {peaks.get('hbm_gbs')} GB/s from "
                                     f"{peak_src})"),
                     "traffic": traffic,
                     "traffic_note": "bytes per launch (mean over the sweep), scaled from the "
                                     "ncu capture at Ng = 64000 by rows x solved columns"},
        "e2e": {"value": replica_value(world, e2e_steps, e2e_ms), "unit": "solves/s",
                "h2d_bytes_per_step": int(h_psi.numel() * 8),
                "d2h_bytes_per_step": int(h_theta.numel() * 8 + piv.nbytes)},
        "gpu_launches": int(sum(launches)),
        "clocks": clk.summary(),
    }
    if world == 1 and not args.no_cpu_baseline:
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


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", choices=["si8", "si64", "si216", "si64c"], default="si64")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--stage", choices=["solve", "select"], default="solve",
                    help="select: time the K-means selection alone (profiling aid)")
    args = ap.parse_args()
    from libisdf_b200 import synth

    shape = synth.SHAPES[args.config]
    if args.impl == "reference":
        run_reference(args, shape)
    elif args.stage == "select":
        run_select(args, shape)
    else:
        run_ours(args, shape)


if __name__ == "__main__":
    main()
