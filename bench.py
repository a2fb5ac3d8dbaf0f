"""ISDF solves/s on B200 (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--config si216|si64|si8] [--precision mixed|fp64]

A step is one full ISDF solve (weight -> K-means selection -> Z C^T GEMM with
the Hadamard epilogue -> C C^T -> Cholesky -> triangular solves) through the
public API, check = false, on synthetic Kohn-Sham-like orbitals of the
configured shape (libisdf_b200/synth.py, seeded per configuration).

Default: the headline comparison, the Si216-like shape (108^3 grid, 864
states, S1 = S2 = all states, mu = 4320, 100 K-means iterations, seed 3) in
the mixed-precision form (value) and in the plain FP64 form of the same run
(plain_fp64, mixed_over_plain), each timed over its own region with its own
clock record, both checked against the oracle's FP64 fit on sampled grid rows
and state pairs (accuracy_vs_oracle); beside them a short Si64-like plain
FP64 run (secondary).

value: solves/s with psi resident in HBM (device time, CUDA events on the
solve stream; max over ranks). e2e: the same through the public API from
host buffers, with the H2D copy of psi and the D2H copy of theta inside the
timed region. Under torchrun each rank runs independent solves on its own GPU
(the path does not shard: replicas only, weak scaling, no collective on the
data path).

--impl reference times the reference's own CPU implementation
(oracle/_ref: the reference sources compiled with single-rank shims) on a
bounded sample of the same workload and extrapolates to solves/s (the line
says so); it also times one whole reference solve at the Si8-like size beside
the model's estimate of it, and the model's scaling with the sampled points.
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


SEEDS = {"si8": 0, "si64": 1, "si216": 3, "si64c": 1, "si216c": 3, "si64vc": 1}  # the benchmark configurations' seeds


def _shape_psi(synth, shape, name):
    """Synthetic orbitals of a workload on the GPU, returned on the host."""
    import torch

    dev = "cuda" if torch.cuda.is_available() else "cpu"
    return synth.shape_orbitals(shape, SEEDS.get(name, 1), device=dev)


# ------------------------------------------------------------------ reference arm
def _slab(shape, mu):
    """A z-slab of the grid with enough points that the reference's Npt x mu
    distance matrix (0.5 GB at least) no longer fits in the host caches, so
    that its cost per point is the full grid's; the whole grid when that is
    smaller."""
    per_plane = shape.n * shape.n
    pts = max(shape.ng // 64, (1 << 29) // (8 * mu))
    nz = min(shape.n, -(-pts // per_plane))
    return nz


def _slab_grid(shape, nz):
    return ((shape.n, shape.n, nz), (shape.length, shape.length, shape.length * nz / shape.n),
            shape.n * shape.n * nz)


def _kmean_model(w, g, ln, mu, best_of=2):
    """(fixed s, s per Lloyd iteration) of the reference's KMEAN on a grid,
    from its whole-routine time with 1 and 3 iterations."""
    from oracle import ref

    t1 = min(ref.bench_kmean(w, g, ln, mu, 1) for _ in range(best_of))
    t3 = min(ref.bench_kmean(w, g, ln, mu, 3) for _ in range(best_of))
    per_iter = max(0.0, (t3 - t1) / 2)
    return max(0.0, t1 - per_iter), per_iter


def calibrate(shape, w):
    """The split of the reference's KMEAN time into a fixed part and a part
    per Lloyd iteration, on the sampled slab (done once per run)."""
    nz = _slab(shape, shape.mu)
    g, ln, npl = _slab_grid(shape, nz)
    fixed, per_iter = _kmean_model(w[:npl], g, ln, shape.mu)
    return {"planes": nz, "fixed_s": fixed, "per_iteration_s": per_iter}


def reference_sample(shape, psi, w, iters: int, cal):
    """Seconds per solve of the reference's CPU path (oracle/_ref: its own
    sources), extrapolated from a bounded sample:
      * K-means: the reference's whole KMEAN (utility.cpp:631-988: filter,
        initial assignment, each Lloyd iteration with its host centroid
        update, pdist2 and findMin, the final argmin, the piv build) with one
        Lloyd iteration on a z-slab of the grid, scaled to `iters` iterations
        by the slab's calibrated split (KMEAN with 1 and 3 iterations:
        fixed part + part per iteration) and to the whole grid by the slab's
        share of the points (the work is Npt x mu per pass);
      * fit: the reference's getbasis_MPI on the same share of the grid rows
        with the full mu, scaled by the rows.
    Returns (seconds per solve, info)."""
    from oracle import ref

    nz = cal["planes"]
    frac = nz / shape.n
    g, ln, npl = _slab_grid(shape, nz)
    t1 = ref.bench_kmean(w[:npl], g, ln, shape.mu, 1)
    fixed, per = cal["fixed_s"], cal["per_iteration_s"]
    scale = (fixed + iters * per) / (fixed + per) if fixed + per > 0 else 1.0
    t_kmeans = t1 * scale / frac
    rows = npl if nz < shape.n else shape.ng
    t_fit = ref.bench_getbasis_rows(psi, shape, shape.ng // rows) * (shape.ng / rows)
    info = {"kind": "reference", "cores": os.cpu_count(), "extrapolated": nz < shape.n,
            "sample": (f"{shape.name}: the reference's KMEAN with one Lloyd iteration on {nz} "
                       f"of {shape.n} z-planes ({npl} points x {shape.mu} centroids), scaled "
                       f"to {iters} iterations by the calibrated split ({fixed:.3f} s fixed + "
                       f"{per:.3f} s per iteration on that slab) and to the whole grid by "
                       f"points; the reference's getbasis_MPI on {rows} of {shape.ng} rows, "
                       f"scaled by rows; OpenBLAS threads = {os.cpu_count()}, K-means "
                       "single-threaded as in the reference"),
            "kmeans_s": t_kmeans, "fit_s": t_fit, "calibration": cal}
    return t_kmeans + t_fit, info


def extrapolation_check(shape, w):
    """Two checks of the sampling model, reported beside its estimate:
      * one whole reference CPU solve at the Si8-like size (40^3, mu = 320,
        100 K-means iterations) timed end to end, beside the model's estimate
        of it (KMEAN with 1 and 3 iterations and getbasis_MPI on the same
        grid): the fixed + per-iteration split;
      * at the workload's own size, the per-iteration time on the sampled
        slab and on a slab twice as thick: the scaling with the points."""
    import time

    from oracle import port, ref
    from libisdf_b200 import synth

    s = synth.SI8
    psi = _shape_psi(synth, s, "si8")
    a = (s.nocc, s.nv1, s.nc1, s.nv2, s.nc2)
    t0 = time.perf_counter()
    piv, rk, it, _ = ref.kmeans_piv(psi, (s.n,) * 3, (s.length,) * 3, *a, s.mu, s.kmeans_iters)
    ref.getbasis(psi, (s.n,) * 3, (s.length,) * 3, *a, rk, piv)
    t_full = time.perf_counter() - t0
    w8 = port.weight(psi, *a)
    fixed, per_iter = _kmean_model(w8, (s.n,) * 3, (s.length,) * 3, s.mu)
    est = fixed + it * per_iter + ref.bench_getbasis_rows(psi, s, 1)
    out = {"si8_whole_solve": {"measured_s": t_full, "model_estimate_s": est,
                               "kmeans_iters": it}}
    nz = _slab(shape, shape.mu)
    if 2 * nz <= shape.n:
        per = []
        for z in (nz, 2 * nz):
            g, ln, npl = _slab_grid(shape, z)
            per.append(_kmean_model(w[:npl], g, ln, shape.mu, best_of=1)[1])
        out["slab_scaling"] = {"planes": [nz, 2 * nz], "s_per_iteration": per,
                               "ratio": per[1] / per[0] if per[0] > 0 else None,
                               "expected_ratio": 2.0}
    return out


def run_reference(args, shape):
    rank, world, _ = _rank_env()
    if rank != 0:
        return
    from oracle import port, ref
    from libisdf_b200 import synth

    if not ref.available():
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref/libisdf_ref.so not built (needs the reference checkout)"}))
        return
    psi = _shape_psi(synth, shape, args.config)
    w = port.weight(psi, shape.nocc, shape.nv1, shape.nc1, shape.nv2, shape.nc2)
    cal = calibrate(shape, w)
    for _ in range(args.warmup):
        reference_sample(shape, psi, w, shape.kmeans_iters, cal)
    times = []
    info = None
    for _ in range(args.steps):
        t, info = reference_sample(shape, psi, w, shape.kmeans_iters, cal)
        times.append(t)
    t = float(np.mean(times))
    v = 1.0 / t
    line = {"metric": METRIC, "value": v, "unit": "solves/s", "impl": "reference",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": _config(shape, args),
            "extrapolated": bool(info["extrapolated"]),
            "cpu_baseline": dict(info, value=v, unit="solves/s"),
            "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    if not args.no_cpu_check:
        line["extrapolation_check"] = extrapolation_check(shape, w)
    print(json.dumps(line), flush=True)


def _config(shape, args, rep=None):
    c = {"workload": shape.name, "ng": shape.ng, "nstate": shape.nstate, "mu": shape.mu,
         "kmeans_iters_cap": shape.kmeans_iters, "selector": args.selector,
         "precision": args.precision, "seed": SEEDS.get(args.config, 1)}
    if args.selector == "qrcp":
        c.update(qrcp_oversample=args.qrcp_factor, qrcp_seed=args.qrcp_seed)
    if args.precision == "mixed":
        c["mixed_slices"] = args.mixed_slices
    if rep is not None:
        c.update(rk_eff=rep.rk_eff, kmeans_iters=rep.kmeans_iters, npt=rep.npt,
                 kmeans_search_frac=round(float(rep.kmeans_search_frac), 4))
    return c


def accuracy_vs_oracle(shape, psi, th_rows, rows, piv, rk, pairs_i, pairs_j, oracle_rows=None):
    """Relative Frobenius error of theta and of the fitted pair densities
    theta C on sampled grid rows and state pairs against the oracle's FP64 fit
    of the same rows (oracle.fit.getbasis_rows: those rows of the full-size
    fit, given the same pivots)."""
    from oracle import fit as ofit

    a = (shape.nocc, shape.nv1, shape.nc1, shape.nv2, shape.nc2)
    th_o = oracle_rows if oracle_rows is not None else ofit.getbasis_rows(psi, *a, rk, piv, rows)
    pm = psi[np.asarray(piv[:rk], dtype=np.int64)]
    C = pm[:, pairs_i] * pm[:, pairs_j]
    fd, fd_o = th_rows[:, :rk] @ C, th_o @ C
    return {"fitted_densities_rel": float(np.linalg.norm(fd - fd_o) / np.linalg.norm(fd_o)),
            "theta_rel": float(np.linalg.norm(th_rows[:, :rk] - th_o) / np.linalg.norm(th_o)),
            "rows": int(len(rows)), "pairs": int(len(pairs_i)),
            "against": "the oracle's FP64 fit (numpy restatement of getbasis_MPI) on those rows"}, th_o


# ------------------------------------------------------------------ our arm
class Timed:
    """K solves on `stream` between two CUDA events, with per-solve events,
    the library's stage times and an nvidia-smi clock record over the region."""

    def __init__(self, torch, solve, stream, steps, device_index, dist=None):
        lat, stage, launches = [], [], []
        with ClockSampler(device_index) as clk:
            e_start = torch.cuda.Event(enable_timing=True)
            e_end = torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            if dist:
                dist.barrier()
            e_start.record(stream)
            for _ in range(steps):
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
        self.t_ms = max_over_ranks(e_start.elapsed_time(e_end), dist, "cuda")
        self.steps = steps
        self.rep = rep
        self.lat = lat
        self.launches = int(sum(launches))
        self.clocks = clk.summary()
        med = lambda k: float(np.median([s_[k] for s_ in stage]))  # noqa: E731
        self.stages = {"select_wall": med(0), "fit_wall": med(1), "zct_gemm": med(3),
                       "cct_cholesky": med(4), "triangular_solve": med(2),
                       "triangular_gemms": med(5)}

    def summary(self, world):
        return {"value": replica_value(world, self.steps, self.t_ms), "unit": "solves/s",
                "steps": self.steps, "ms_per_step": self.t_ms / self.steps,
                "latency_ms": {"p50": float(np.percentile(self.lat, 50)),
                               "p99": float(np.percentile(self.lat, 99))},
                "stages_ms": self.stages, "clocks": self.clocks}


def _e2e(torch, solve, stream, d_psi, d_theta, h_psi, steps, dist):
    """End to end from host buffers, as a caller that consumes theta on the
    host runs it: every step copies its psi in (pinned host -> HBM), solves,
    and copies theta out (HBM -> pinned host), in a steady pipeline: the psi
    of step i+1 is copied in on an H2D stream and the theta of step i copied
    out on a D2H stream while step i+1 solves (two device psi and theta
    buffers when HBM allows, else one of each and those copies do not
    overlap). Returns (ms, theta buffers, psi buffers, D2H bytes per step)."""
    h_theta = torch.empty(d_theta.shape, dtype=torch.float64).pin_memory()
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
    done = [None] * len(thetas)  # theta buffer copied out
    used = [None] * len(psis)    # psi buffer no longer read by a solve
    ready = [None] * len(psis)   # psi buffer holds its step's input

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
    for i in range(steps):
        pb, tb = i % len(psis), i % len(thetas)
        stream.wait_event(ready[pb])
        if done[tb] is not None:
            stream.wait_event(done[tb])
        if len(psis) > 1 and i + 1 < steps:
            fetch(i + 1)  # into the other buffer, beside this solve
        solve(thetas[tb], psis[pb])
        solved = torch.cuda.Event()
        solved.record(stream)
        used[pb] = solved
        if len(psis) == 1 and i + 1 < steps:
            fetch(i + 1)
        copy_stream.wait_event(solved)
        with torch.cuda.stream(copy_stream):
            # in 256 MB pieces, so that the library's small state reads of the
            # next solve are not queued behind one long copy
            src, dst = thetas[tb].view(-1), h_theta.view(-1)
            piece = 1 << 25
            for o in range(0, src.numel(), piece):
                dst[o:o + piece].copy_(src[o:o + piece], non_blocking=True)
        done[tb] = torch.cuda.Event()
        done[tb].record(copy_stream)
    stream.wait_stream(copy_stream)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1), dist, "cuda")
    nb = (len(thetas), len(psis), int(h_theta.numel() * 8))
    del thetas, psis, h_theta
    return (ms,) + nb


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
    psi = _shape_psi(synth, shape, args.config)
    ng, mu = shape.ng, shape.mu
    h_psi = torch.from_numpy(np.ascontiguousarray(psi.T)).pin_memory()
    d_psi = h_psi.cuda()
    d_theta = torch.empty((mu, ng), dtype=torch.float64, device="cuda")
    piv = np.zeros(ng, dtype=np.int32)
    dom = isdf.Domain(length=(shape.length,) * 3, num_grid=(shape.n,) * 3)
    stream = torch.cuda.Stream()
    s1 = "QRCP" if args.selector == "qrcp" else "Kmeans"
    mixed = args.precision == "mixed"
    compare = mixed and not args.no_compare

    def options(prec):
        return isdf.Options(stream=stream.cuda_stream, precision=prec,
                            qrcp_oversample=args.qrcp_factor, qrcp_seed=args.qrcp_seed,
                            mixed_slices=args.mixed_slices)

    opts = options(isdf.PRECISION_MIXED if mixed else isdf.PRECISION_FP64)
    opts64 = options(isdf.PRECISION_FP64)

    def solve(theta=None, psi_d=None, o=None):
        return isdf.ISDF(d_psi if psi_d is None else psi_d, dom, shape.nocc, shape.nstate,
                         shape.nv1, shape.nc1, shape.nv2, shape.nc2, mu,
                         d_theta if theta is None else theta, piv, shape.kmeans_iters, s1=s1,
                         options=o or opts)

    fp64_peak = _fp64_peak_tflops(torch)
    int8_peak = _int8_peak_tops(torch) if mixed else None
    rng = np.random.default_rng(0)
    rows = np.sort(rng.choice(ng, size=min(2048, ng), replace=False))
    pi = shape.nocc - shape.nv1 + rng.integers(0, shape.nv1 + shape.nc1, size=1024)
    pj = shape.nocc - shape.nv2 + rng.integers(0, shape.nv2 + shape.nc2, size=1024)
    d_rows = torch.from_numpy(rows).cuda()

    def theta_rows(rk):
        return d_theta[:rk].index_select(1, d_rows).T.cpu().numpy()

    with torch.cuda.stream(stream):
        for _ in range(max(3, args.warmup)):
            solve()
        main = Timed(torch, solve, stream, args.steps, local, dist)
        rep = main.rep
        rk = rep.rk_eff
        th_main = theta_rows(rk) if rank == 0 else None
        piv_main = piv[:rk].copy()
        plain = None
        if compare:
            solve64 = lambda: solve(o=opts64)  # noqa: E731
            for _ in range(3):
                solve64()
            plain = Timed(torch, solve64, stream, max(3, min(args.steps, 8)), local, dist)
            th_plain = theta_rows(rk) if rank == 0 else None
            assert np.array_equal(piv[:rk], piv_main), "piv differs between the forms"
        if dist:
            dist.barrier()
        e2e_steps = max(8, args.steps)
        e2e_ms, e2e_bufs, e2e_psi_bufs, d2h_theta = _e2e(
            torch, lambda th, ps: solve(th, ps), stream, d_psi, d_theta, h_psi, e2e_steps, dist)
    if dist:
        dist.destroy_process_group()
    if rank != 0:
        return
    accuracy = {}
    acc_main, th_o = accuracy_vs_oracle(shape, psi, th_main, rows, piv_main, rk, pi, pj)
    accuracy["mixed" if mixed else "fp64"] = acc_main
    if plain is not None:
        accuracy["fp64"], _ = accuracy_vs_oracle(shape, psi, th_plain, rows, piv_main, rk, pi,
                                                 pj, th_o)
    peaks, peak_src = _measured_peaks()
    v = replica_value(world, args.steps, main.t_ms)
    S = args.mixed_slices
    gemm_ms = main.stages["triangular_gemms"]
    solve_ms = (plain or main).stages["triangular_solve"]
    roof64 = None
    if plain is not None or not mixed:
        # k_trsm_ws, the two triangular sweeps of the FP64 form as in-place FP64
        # tensor-core GEMMs: 2*Ng*rk^2 flops per solve over the stage's
        # CUDA-event time (the k_trsm_ws launches plus the small k_build_w
        # launches between them, so a slight underestimate of the kernel's
        # own rate). DRAM traffic per launch: 8.40 B per grid row and solved
        # column (ncu on the 40^3-grid case) x the mean solved width (rk/2 + 32).
        ach = 2.0 * ng * rk * rk / (solve_ms * 1e-3) / 1e12 if solve_ms > 0 else None
        roof64 = {"kernel": "k_trsm_ws (both sweeps of the FP64 triangular solve)",
                  "bound": "tensor", "achieved": ach, "peak": fp64_peak, "unit": "TFLOP/s",
                  "frac": (ach / fp64_peak) if ach else None,
                  "peak_source": ("cuBLAS DGEMM 8192^3 measured in this run: the FP64 "
                                  "denominator (the measured-peaks file holds HBM and BF16 "
                                  f"figures only; HBM {peaks.get('hbm_gbs')} GB/s from "
                                  f"{peak_src})"),
                  "traffic": 8.40 * ng * (rk / 2 + 32),
                  "traffic_note": "bytes per launch (mean over the sweep), scaled from the "
                                  "ncu capture at Ng = 64000 by rows x solved columns"}
    if mixed:
        # k_ozaki_gemm, the two triangular products Y = Z L^-T and theta = Y L^-1
        # as INT8 digit-pair GEMMs: issued INT8 ops per solve 2 GEMMs x 2 x Ng x
        # rk x (rk/2 + 32) x S(S+1)/2 (each tile runs the K range its triangular
        # factor leaves nonzero), over CUDA events around the two launches.
        ops = 2 * 2.0 * ng * rk * (rk / 2 + 32) * S * (S + 1) / 2
        ach = ops / (gemm_ms * 1e-3) / 1e12 if gemm_ms > 0 else None
        # DRAM traffic per launch from ncu on the 40^3-grid case (Ng = 64000,
        # rk = 4312, S = 6; mean of the two products): 8.855 GB read (the
        # digits of both operands, B's re-read once per raster group, so
        # ~ rows x rk^2) and 2.195 GB written (the FP64 output, rows x rk).
        # Reported only near that shape, where the scaling holds.
        if S == 6 and 0.8 <= rk / 4312 <= 1.25:
            traffic = (8.855e9 * (ng / 64000) * (rk / 4312) ** 2 +
                       2.195e9 * (ng / 64000) * (rk / 4312))
            traffic_note = ("bytes per launch (mean of the two products), scaled from the ncu "
                            "capture at Ng = 64000, rk = 4312: reads by rows x rk^2, writes "
                            f"by rows x rk; algorithmic {(ng * rk * (S + 8)) / 1e9:.1f} GB")
        else:
            traffic, traffic_note = None, "no ncu capture at this rk and S"
        roofline = {"kernel": "k_ozaki_gemm (Y = Z L^-T and theta = Y L^-1, INT8 digit pairs)",
                    "bound": "tensor", "achieved": ach, "peak": int8_peak[0],
                    "unit": "TOPS (INT8)", "frac": (ach / int8_peak[0]) if ach else None,
                    "peak_burst": int8_peak[1],
                    "frac_of_burst": (ach / int8_peak[1]) if ach else None,
                    "peak_source": int8_peak[2],
                    "emulated_fp64_tflops": (2.0 * 2 * ng * rk * (rk / 2 + 32) /
                                             (gemm_ms * 1e-3) / 1e12) if gemm_ms > 0 else None,
                    "traffic": traffic, "traffic_note": traffic_note}
    else:
        roofline = roof64
    line = {
        "metric": METRIC, "value": v, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": max(3, args.warmup), "ms_per_step": main.t_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": dict(_config(shape, args, rep), parallelism=f"replicas x{world}",
                       l2=(f"inputs larger than L2 (psi {ng * shape.nstate * 8 / 1e9:.2f} GB, "
                           f"theta {ng * mu * 8 / 1e9:.2f} GB; L2 126 MB)")),
        "latency_ms": main.summary(world)["latency_ms"],
        "stages_ms": main.stages,
        "roofline": roofline,
        "e2e": {"value": replica_value(world, e2e_steps, e2e_ms), "unit": "solves/s",
                "h2d_bytes_per_step": int(h_psi.numel() * 8),
                "d2h_bytes_per_step": int(d2h_theta + piv.nbytes),
                "steps": e2e_steps, "theta_buffers": e2e_bufs, "psi_buffers": e2e_psi_bufs,
                "form": args.precision},
        "gpu_launches": main.launches,
        "accuracy_vs_oracle": accuracy,
        "clocks": main.clocks,
    }
    if plain is not None:
        p = plain.summary(world)
        line["plain_fp64"] = dict(p, roofline=roof64)
        line["mixed_over_plain"] = v / p["value"]
    if not args.no_secondary and shape is not synth.SI64 and world == 1:
        # the headline's buffers go first (the solve closures hold them)
        d_psi = d_theta = h_psi = d_rows = None
        line["secondary"] = secondary_si64(torch, isdf, synth, fp64_peak)
    if world == 1 and not args.no_cpu_baseline and s1 == "QRCP":
        line["cpu_baseline"] = {"value": None, "unit": "solves/s",
                                "unavailable": "the reference's QRCP selector runs ScaLAPACK "
                                               "pdgeqpf, which cannot be built here"}
    elif world == 1 and not args.no_cpu_baseline:
        try:
            from oracle import port

            w = port.weight(psi, shape.nocc, shape.nv1, shape.nc1, shape.nv2, shape.nc2)
            t_cpu, info = reference_sample(shape, psi, w, rep.kmeans_iters, calibrate(shape, w))
            line["cpu_baseline"] = dict(info, value=1.0 / t_cpu, unit="solves/s")
        except Exception as e:  # the reference build is optional on the box
            line["cpu_baseline"] = {"value": None, "unit": "solves/s",
                                    "unavailable": str(e)[:200]}
    print(json.dumps(line), flush=True)


def secondary_si64(torch, isdf, synth, fp64_peak):
    """The Si64-like plain FP64 solve (80^3, 256 states, mu = 2048, K-means),
    a short run beside the headline: solves/s, stages and clocks."""
    torch.cuda.empty_cache()
    s = synth.SI64
    psi = _shape_psi(synth, s, "si64")
    d_psi = torch.from_numpy(np.ascontiguousarray(psi.T)).cuda()
    d_theta = torch.empty((s.mu, s.ng), dtype=torch.float64, device="cuda")
    piv = np.zeros(s.ng, dtype=np.int32)
    dom = isdf.Domain(length=(s.length,) * 3, num_grid=(s.n,) * 3)
    stream = torch.cuda.Stream()
    opts = isdf.Options(stream=stream.cuda_stream)

    def solve():
        return isdf.ISDF(d_psi, dom, s.nocc, s.nstate, s.nv1, s.nc1, s.nv2, s.nc2, s.mu, d_theta,
                         piv, s.kmeans_iters, options=opts)

    with torch.cuda.stream(stream):
        for _ in range(3):
            solve()
        t = Timed(torch, solve, stream, 5, 0)
    out = t.summary(1)
    rk = t.rep.rk_eff
    ms = out["stages_ms"]["triangular_solve"]
    ach = 2.0 * s.ng * rk * rk / (ms * 1e-3) / 1e12 if ms > 0 else None
    out.update(workload=s.name, precision="fp64", rk_eff=rk, kmeans_iters=t.rep.kmeans_iters,
               roofline={"kernel": "k_trsm_ws", "achieved": ach, "peak": fp64_peak,
                         "unit": "TFLOP/s", "frac": (ach / fp64_peak) if ach else None})
    return out


def _int8_peak_tops(torch):
    """cuBLASLt INT8 GEMM (torch._int_mm, 8192^3): the INT8 tensor-core
    denominator for the mixed form's GEMMs, measured as a burst (best of 5)
    and sustained (back to back for ~3 s, under the power cap, the condition
    the mixed form's products run in inside a solve). Returns (sustained TOPS,
    burst TOPS, source)."""
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
        burst = 2 * 8192 ** 3 / (best * 1e-3) / 1e12
        n = max(8, int(3.0 / (best * 1e-3)))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(n):
            torch._int_mm(a, b)
        e1.record()
        torch.cuda.synchronize()
        sustained = n * 2 * 8192 ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12
        del a, b
        torch.cuda.empty_cache()
        return sustained, burst, ("cuBLASLt INT8 GEMM 8192^3 measured in this run, back to back "
                                  f"for ~3 s ({n} GEMMs; the burst best of 5: {burst:.0f} TOPS)")
    except Exception as e:  # noqa: BLE001
        peaks, _ = _measured_peaks()
        return (2.0 * peaks["bf16_tflops_sustained"], 2.0 * peaks["bf16_tflops"],
                f"2 x measured dense BF16 (INT8 GEMM unavailable: {e})")



def run_select(args, shape):
    """--stage select: the K-means selection alone (weight computed once),
    selections/s; a small-footprint command for profiling the K-means kernels
    at full grid size (psi, the weight and the K-means workspace only).
    With --batch B > 1: B systems of the shape (seeds 100..), their selections
    in one batched launch (isdf_kmeans_select_batch) against the same B run
    one after another through isdf_kmeans_select, both timed."""
    import torch

    import libisdf_b200 as isdf
    from libisdf_b200 import synth

    torch.cuda.set_device(0)
    B = max(1, args.batch)
    dom = isdf.Domain(length=(shape.length,) * 3, num_grid=(shape.n,) * 3)
    stream = torch.cuda.Stream()
    ws = []
    for b in range(B):
        psi = synth.shape_orbitals(shape, 1 if B == 1 else 100 + b, device="cuda")
        d_psi = torch.from_numpy(np.ascontiguousarray(psi.T)).cuda()
        d_w = torch.empty(shape.ng, dtype=torch.float64, device="cuda")
        isdf.kmeans_weight(d_psi, shape.ng, shape.nstate, shape.nocc, shape.nv1, shape.nc1,
                           shape.nv2, shape.nc2, d_w, stream=stream.cuda_stream)
        ws.append(d_w)
        del d_psi
    torch.cuda.synchronize()

    def one_by_one():
        out = []
        for d_w in ws:
            out.append(isdf.kmeans_select(dom, d_w, shape.mu, shape.kmeans_iters,
                                          stream=stream.cuda_stream))
        return out

    def batched():
        return isdf.kmeans_select_batch([dom] * B, ws, [shape.mu] * B,
                                        [shape.kmeans_iters] * B, stream=stream.cuda_stream)

    def timed(fn):
        for _ in range(max(3, args.warmup)):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            out = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1), out

    t_ms, out = timed(one_by_one)
    line = {"metric": "K-means selections/s", "value": B * args.steps / (t_ms * 1e-3),
            "unit": "selections/s", "n_gpus": 1, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": t_ms / args.steps,
            "higher_is_better": True, "dtype": "f64", "data": "synthetic",
            "config": {"workload": shape.name, "ng": shape.ng, "mu": shape.mu,
                       "systems_per_step": B, "rk_eff": out[0][1], "kmeans_iters": out[0][2],
                       "npt": out[0][3]}}
    if B > 1:
        tb_ms, outb = timed(batched)
        same = all(np.array_equal(a[0], b[0]) and a[1:] == b[1:] for a, b in zip(out, outb))
        line["batched"] = {"value": B * args.steps / (tb_ms * 1e-3), "unit": "selections/s",
                           "ms_per_step": tb_ms / args.steps, "identical_to_one_by_one": same,
                           "speedup": t_ms / tb_ms}
    print(json.dumps(line), flush=True)


def run_sharded(args, shape):
    """--shard: one system split by grid rows over the ranks torchrun starts
    (the reference's p-rank layout; NCCL between the GPUs, its id handed out
    over the torch process group). Strong scaling: every step is one solve of
    the whole system; value = steps / (max over ranks of the timed region)."""
    import datetime

    import torch
    import torch.distributed as tdist

    import libisdf_b200 as isdf
    from libisdf_b200 import synth

    rank, world, local = _rank_env()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                 device_id=torch.device("cuda", local))
        dist = tdist
    psi = _shape_psi(synth, shape, args.config)
    ng, mu = shape.ng, shape.mu
    start, cnt = isdf.row_block(ng, world, rank)
    d_rows = torch.from_numpy(np.ascontiguousarray(psi[start:start + cnt].T)).cuda()
    del psi
    layout = isdf.THETA_CYCLIC if args.theta_layout == "cyclic" else isdf.THETA_ROWS
    width = mu // world + (1 if rank < mu % world else 0)
    d_theta = (torch.empty((width, ng), dtype=torch.float64, device="cuda")
               if layout == isdf.THETA_CYCLIC else
               torch.empty((mu, cnt), dtype=torch.float64, device="cuda"))
    piv = np.zeros(ng, dtype=np.int32)
    dom = isdf.Domain(length=(shape.length,) * 3, num_grid=(shape.n,) * 3)
    comm = (isdf.Comm.nccl_from_torch() if dist else
            isdf.Comm.nccl(isdf.nccl_unique_id(), 0, 1))
    stream = torch.cuda.Stream()
    prec = isdf.PRECISION_MIXED if args.precision == "mixed" else isdf.PRECISION_FP64
    opts = isdf.Options(stream=stream.cuda_stream, precision=prec, mixed_slices=args.mixed_slices)

    def solve():
        return isdf.solve_sharded(comm, d_rows, dom, shape.nocc, shape.nstate, shape.nv1,
                                  shape.nc1, shape.nv2, shape.nc2, mu, d_theta, piv,
                                  shape.kmeans_iters, layout=layout, options=opts)

    with torch.cuda.stream(stream):
        for _ in range(max(3, args.warmup)):
            solve()
        main = Timed(torch, solve, stream, args.steps, local, dist)
    t_ms = main.t_ms
    if rank == 0:
        line = {"metric": METRIC, "value": args.steps / (t_ms * 1e-3), "unit": "solves/s",
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": t_ms / args.steps, "higher_is_better": True, "scaling": "strong",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": dict(_config(shape, args, main.rep), parallelism=f"shard{world}",
                               theta_layout=args.theta_layout),
                "stages_ms": main.stages, "gpu_launches": main.launches,
                "clocks": main.clocks}
        print(json.dumps(line), flush=True)
    comm.close()
    if dist:
        tdist.barrier()
        tdist.destroy_process_group()


def _serve_setup(args, torch, isdf, synth):
    """psi pools per shape (seeds 100, 101, ...) and theta buffers, on the GPU."""
    shapes = [synth.SI8, synth.SI64, synth.SI216]
    pool_seeds = [4, 2, 1]
    theta_bufs = [16, 3, 1]
    mix = [0.6, 0.3, 0.1]
    if args.serve_mix != "standard":
        # one shape only (the served form's throughput at that size)
        k1 = {"si8": 0, "si64": 1, "si216": 2}[args.serve_mix]
        mix = [1.0 if k == k1 else 0.0 for k in range(3)]
        pool_seeds = [1 if k == k1 else 0 for k in range(3)]
        # in flight: the slots' requests plus a batch of small ones
        inflight = args.slots + (args.batch_small if k1 == 0 else 0)
        theta_bufs = [inflight if k == k1 else 0 for k in range(3)]
    psi = {k: [torch.from_numpy(np.ascontiguousarray(
        synth.shape_orbitals(shapes[k], 100 + j, device="cuda").T)).cuda()
        for j in range(pool_seeds[k])] for k in range(3)}
    thetas = {k: [torch.empty((shapes[k].mu, shapes[k].ng), dtype=torch.float64, device="cuda")
                  for _ in range(theta_bufs[k])] for k in range(3)}
    doms = [isdf.Domain(length=(sh.length,) * 3, num_grid=(sh.n,) * 3) for sh in shapes]
    torch.cuda.synchronize()
    return shapes, pool_seeds, theta_bufs, mix, psi, thetas, doms


def serve_once(args, torch, isdf, setup, rate, precision, batch_small):
    """One pass of args.requests Poisson arrivals at `rate` requests/s through
    a fresh server. Latency is arrival -> completion as the client sees it
    (it includes any wait for a free output buffer); throughput is requests /
    (last completion - first arrival)."""
    shapes, pool_seeds, theta_bufs, mix, psi, thetas, doms = setup
    rng = np.random.default_rng(args.serve_seed)
    n_req = args.requests
    kinds = rng.choice(3, size=n_req, p=mix)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=n_req))
    prec = isdf.PRECISION_MIXED if precision == "mixed" else isdf.PRECISION_FP64
    opts = isdf.Options(precision=prec)
    free = {k: list(thetas[k]) for k in range(3)}
    budget = 0
    if args.hbm_budget_gb > 0:
        budget = int(args.hbm_budget_gb * (1 << 30))
    elif args.hbm_budget_gb < 0:  # all that is free now, less 4 GiB
        budget = max(0, torch.cuda.mem_get_info()[0] - (4 << 30))
    srv = isdf.Server(slots=args.slots, hbm_budget_bytes=budget, batch_small=batch_small)
    lock = threading.Condition()
    inflight = {}  # ticket -> (kind, theta, arrival index)
    done_at = np.zeros(n_req)
    errors = []

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
                            errors.append(t)
                    lock.notify_all()
            time.sleep(0.0005)

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
    return {"rate_per_s": rate, "precision": precision, "batch_small": batch_small,
            "solves_per_s": n_req / span, "kept_up": bool(n_req / span >= 0.95 * rate),
            "latency_ms": {"p50": float(np.percentile(lat, 50)),
                           "p99": float(np.percentile(lat, 99)),
                           "p50_by_shape": {shapes[k].name: float(np.percentile(lat[kinds == k], 50))
                                            for k in range(3) if (kinds == k).any()},
                           "p99_by_shape": {shapes[k].name: float(np.percentile(lat[kinds == k], 99))
                                            for k in range(3) if (kinds == k).any()}},
            "errors": len(errors),
            "server": {k: stats[k] for k in stats if k in ("completed", "peak_concurrency",
                                                              "p50_ms", "p99_ms", "peak_bytes")},
            "clocks": clk.summary()}


def run_serve(args):
    """--serve: the serving mix (60 % Si8-like, 30 % Si64-like, 10 % Si216-like
    requests, K-means; per-request orbitals from a small pool of seeds per
    shape, every in-flight request with its own theta and piv) arriving as a
    Poisson process through the continuous-batching server (isdf_server_*),
    at each rate of --rates (default: --rate) and for each form of
    --serve-forms; one JSON line with the whole sweep."""
    import torch

    import libisdf_b200 as isdf
    from libisdf_b200 import synth

    torch.cuda.set_device(0)
    setup = _serve_setup(args, torch, isdf, synth)
    rates = [float(x) for x in args.rates.split(",")] if args.rates else [args.rate]
    forms = args.serve_forms.split(",")
    sweep = [serve_once(args, torch, isdf, setup, r, f, args.batch_small)
             for f in forms for r in rates]
    best = {f: max((x for x in sweep if x["precision"] == f), key=lambda x: x["solves_per_s"])
            for f in forms}
    head = best[forms[0]]
    line = {"metric": "served ISDF solves/s (serving mix)", "value": head["solves_per_s"],
            "unit": "solves/s", "n_gpus": 1, "higher_is_better": True, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": ("serving mix: 60 % Si8-like, 30 % Si64-like, 10 % Si216-like, "
                                    "K-means" if args.serve_mix == "standard" else
                                    f"served {args.serve_mix} requests only, K-means"),
                       "requests_per_rate": args.requests, "rates_per_s": rates,
                       "forms": forms, "slots": args.slots, "batch_small": args.batch_small,
                       "hbm_budget_gb": args.hbm_budget_gb},
            "best_by_form": {f: {"rate_per_s": b["rate_per_s"], "solves_per_s": b["solves_per_s"],
                                 "p50_ms": b["latency_ms"]["p50"],
                                 "p99_ms": b["latency_ms"]["p99"]} for f, b in best.items()},
            "sweep": sweep}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", choices=["si8", "si64", "si216", "si64c", "si216c", "si64vc"],
                    default="si216")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="mixed")
    ap.add_argument("--no-compare", action="store_true",
                    help="mixed precision: skip the plain FP64 run of the same workload")
    ap.add_argument("--no-secondary", action="store_true",
                    help="skip the short Si64-like plain FP64 run beside the headline")
    ap.add_argument("--no-cpu-check", action="store_true",
                    help="reference arm: skip the whole Si8-like reference solve")
    ap.add_argument("--mixed-slices", type=int, choices=[5, 6, 7], default=6,
                    help="INT8 digits per operand in the mixed form (Options.mixed_slices)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--selector", choices=["kmeans", "qrcp"], default="kmeans")
    ap.add_argument("--qrcp-factor", type=float, default=1.5,
                    help="QRCP oversampling (numPre = round(sqrt(f mu)); the reference uses 1.5)")
    ap.add_argument("--qrcp-seed", type=int, default=41)
    ap.add_argument("--stage", choices=["solve", "select"], default="solve",
                    help="select: time the K-means selection alone (profiling aid)")
    ap.add_argument("--batch", type=int, default=1,
                    help="--stage select: systems per step, batched launch vs one by one")
    ap.add_argument("--serve", action="store_true",
                    help="the serving mix through isdf_server_* (Poisson arrivals)")
    ap.add_argument("--requests", type=int, default=512)
    ap.add_argument("--rate", type=float, default=4.0, help="arrivals per second (--serve)")
    ap.add_argument("--rates", type=str, default="",
                    help="--serve: comma-separated arrival rates to sweep (default: --rate)")
    ap.add_argument("--serve-forms", type=str, default="mixed,fp64",
                    help="--serve: comma-separated precisions to serve (mixed, fp64)")
    ap.add_argument("--batch-small", type=int, default=32,
                    help="--serve: small requests per batched K-means launch (0: off)")
    ap.add_argument("--slots", type=int, default=4)
    ap.add_argument("--serve-seed", type=int, default=7)
    ap.add_argument("--serve-mix", choices=["standard", "si8", "si64", "si216"], default="standard",
                    help="standard: 60/30/10 Si8/Si64/Si216; else one shape only")
    ap.add_argument("--shard", action="store_true",
                    help="split one system by grid rows over the ranks (strong scaling) "
                         "instead of one replica per GPU")
    ap.add_argument("--theta-layout", choices=["rows", "cyclic"], default="rows",
                    help="--shard: theta as each rank's rows, or the reference's cyclic columns")
    ap.add_argument("--hbm-budget-gb", type=float, default=-1.0,
                    help="server workspace budget (0: the library default, half the free memory; "
                         "-1: all free memory less 4 GiB once the request buffers are allocated)")
    args = ap.parse_args()
    from libisdf_b200 import synth

    shape = synth.SHAPES[args.config]
    if args.impl == "reference":
        run_reference(args, shape)
    elif args.serve:
        run_serve(args)
    elif args.shard:
        run_sharded(args, shape)
    elif args.stage == "select":
        run_select(args, shape)
    else:
        run_ours(args, shape)


if __name__ == "__main__":
    main()
