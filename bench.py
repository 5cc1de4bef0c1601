"""Benchmark: milliseconds per n = 1788 generalized eigensolve (sygvd, H C = S C e, all eigenpairs) on a B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--n 1788]

Workload: the generalized construction with n = 1788, seed 2 (S = I + banded random overlap with lambda_min >= 0.05,
H = S^1/2 Q diag(lam) Q^T S^1/2, lam ~ U[-1.0, 0.5] Eh with a 0.05 Eh HOMO/LUMO gap at n/2), FP64 throughout on the
GPU (potrf -> X = U^-1 -> X^T H X -> resident sytrd -> divide-and-conquer stedc -> compact-WY ormtr -> X C').
Synthetic seeded inputs stand in for the GFN2 H/S dumps the reference reads (none are published).

ours (default):  one step = restore H, S on the device (D2D copy of pristine inputs) + one device-pointer solve on
    torch's current stream, timed with CUDA events per step; L2 is flushed (256 MB write) before every timed step,
    outside the events.  `value` = mean ms per solve (whole job: summed over replicas for N > 1, because a single
    solve does not shard and the ranks are independent replicas).  `e2e` = the same solve through the C ABI with
    pinned HOST buffers (H2D of H and S, D2H of C, U and e inside the timed region).  `roofline` = the resident
    reduction kernel (sytrd): algorithmic bytes 4 n^3 / 3 (its symv reads n^3/6 FP64 elements) / its event-timed
    duration, against the measured HBM copy bandwidth.  `cpu_baseline` = the reference's LAPACK chain (dpotrf, dsygst,
    dsytrd, dstedc, dormtr, dtrsm from OpenBLAS) on the host cores, rank 0, bounded sample.
reference:  the same LAPACK chain on the host cores only (rank 0; other ranks exit), the reference's CPU path.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "xtb-diagonalization_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)

METRIC = "ms per n=1788 generalized eigensolve (sygvd, all eigenpairs)"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=1788)
    ap.add_argument("--seed", type=int, default=2)
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--cpu-budget-s", type=float, default=20.0, help="bound on the CPU baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--batch-count", type=int, default=256, help="uneven batch size (0: skip the batch section)")
    ap.add_argument("--cpu-batch-sample", type=int, default=256,
                    help="problems of the CPU P x 1 batch protocol in the cpu_baseline leg (0: skip)")
    ap.add_argument("--cpu-protocol", action="store_true",
                    help="only the CPU baseline protocol of every configuration (no GPU): one JSON line")
    ap.add_argument("--batch-steps", type=int, default=3)
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision section")
    ap.add_argument("--no-autotune", action="store_true", help="use the default plan instead of autotuning it")
    ap.add_argument("--no-two-stage", action="store_true", help="skip the two-stage reduction section")
    ap.add_argument("--adjoint-count", type=int, default=32, help="problems of the density-adjoint section (0: skip)")
    ap.add_argument("--hs-bin", default=None, help="solve an H/S dump (hsbin format) instead of the synthetic pair")
    return ap.parse_args()


def rank_info():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0")),
            int(os.environ.get("WORLD_SIZE", "1")))


# ------------------------------------------------------------------------------------------------ inputs

def triangle_bytes(n, block=128):
    """Bytes of one triangle of an n x n FP64 matrix as the library's host-pointer dsygvd moves it: 2D copies of blocks
    of `block` columns, each with the rows 0 .. (block end - 1) (the diagonal blocks travel whole)."""
    return 8 * sum(min(n, c0 + block) * (min(n, c0 + block) - c0) for c0 in range(0, n, block))


def build_generalized(n, seed):
    """The generalized benchmark pair, built on the host with numpy's default_rng(seed) so that both bench arms (the
    GPU path and the CPU LAPACK chain) solve the same bytes: S = I + G (G_ij = 0.35 exp(-|i-j|/12) u_ij, u ~ U[-1, 1]
    drawn as a full n x n matrix of which the strict upper triangle is used, zero diagonal), shifted so that
    lambda_min(S) >= 0.05; lam ~ U[-1.0, 0.5] Eh sorted, lam[n//2:] += 0.05 (the HOMO/LUMO gap); Q from the QR of a
    standard normal n x n matrix (column signs fixed by R's diagonal); H = S^1/2 Q diag(lam) Q^T S^1/2 symmetrised.
    Returns (H, S, lam) with H, S column-major float64 and lam the exact generalized spectrum (ascending).  Input
    generation only, never timed."""
    import numpy as np

    rng = np.random.default_rng(seed)
    idx = np.arange(n)
    dist = np.abs(idx[:, None] - idx[None, :])
    u = rng.uniform(-1.0, 1.0, (n, n))
    g = 0.35 * np.exp(-dist / 12.0) * np.triu(u, 1)
    s = np.eye(n) + g + g.T
    lmin = np.linalg.eigvalsh(s)[0]
    if lmin < 0.05:
        s += (0.05 - lmin) * np.eye(n)
    lam = np.sort(rng.uniform(-1.0, 0.5, n))
    lam[n // 2:] += 0.05
    q, r = np.linalg.qr(rng.standard_normal((n, n)))
    q = q * np.sign(np.diag(r))[None, :]
    ws, vs = np.linalg.eigh(s)
    shalf = (vs * np.sqrt(ws)[None, :]) @ vs.T
    shalf = 0.5 * (shalf + shalf.T)
    h = shalf @ ((q * lam[None, :]) @ q.T) @ shalf
    h = 0.5 * (h + h.T)
    return np.asfortranarray(h), np.asfortranarray(s), lam


def bench_config(n, seed):
    """The `config` object of both arms' lines (identical, so that the two arms are seen to run one workload)."""
    return {"workload": f"generalized eigensolve H C = S C e, n={n}, seed={seed}, all eigenpairs, FP64 "
                        "(potrf, sygst, sytrd, stedc, ormtr, trsm)",
            "inputs": f"host numpy default_rng({seed}) construction (bench.build_generalized), the same bytes in both "
                      "arms",
            "l2": "GPU arm: flushed (256 MB write) before every timed step; CPU arm: n/a"}


def host_cpu():
    """nproc and the CPU model of this host."""
    model = None
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return os.cpu_count(), model


# ------------------------------------------------------------------------------------------------ clocks

class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str):
        self.gpu_id = gpu_id
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", self.gpu_id, f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, ValueError):
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=5)
        sm, smax, power, reasons = [], [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
                power.append(float(parts[3]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm), "power_w_max": max(power) if power else None}


# ------------------------------------------------------------------------------------------------ CPU path

def cpu_chain_time(h, s, budget_s: float, max_runs: int):
    """The reference's LAPACK chain on the host: ms per solve over a bounded sample, and the thread count used."""
    import numpy as np

    from oracle import lapack

    threads = lapack.get_threads()
    times = []
    t_end = time.perf_counter() + budget_s
    while len(times) < max_runs and (not times or time.perf_counter() < t_end):
        t0 = time.perf_counter()
        w, c = lapack.sygvd_chain(h, s)
        times.append((time.perf_counter() - t0) * 1e3)
    assert np.all(np.isfinite(w))
    return statistics.median(times), len(times), threads


def cpu_reference_solution(h, s):
    """The reference's LAPACK chain's (w, C) on the same input (the checker of the GPU arm's accuracy fields)."""
    from oracle import lapack

    return lapack.sygvd_chain(h, s)


def cpu_one_thread_time(h, s, runs=3):
    """The same chain with OpenBLAS on one thread (the reference's single-thread protocol): median ms of `runs` after
    one untimed solve; the thread count is restored afterwards."""
    from oracle import lapack

    t_all = lapack.get_threads()
    lapack.set_threads(1)
    try:
        lapack.sygvd_chain(h, s)
        ts = []
        for _ in range(runs):
            t0 = time.perf_counter()
            lapack.sygvd_chain(h, s)
            ts.append((time.perf_counter() - t0) * 1e3)
    finally:
        lapack.set_threads(t_all)
    return statistics.median(ts), runs


def _cpu_batch_worker(jobs, barrier, out_q):
    """One of P single-thread processes of the CPU batch protocol: builds its problems (untimed), waits for the other
    processes, then solves them one after another with the LAPACK chain on one OpenBLAS thread."""
    os.environ["OPENBLAS_NUM_THREADS"] = "1"
    os.environ["OMP_NUM_THREADS"] = "1"
    for p in (ROOT, PKG):
        if p not in sys.path:
            sys.path.insert(0, p)
    from oracle import lapack

    lapack.set_threads(1)
    probs = [build_generalized(n, seed) for n, seed in jobs]
    barrier.wait()
    t0 = time.perf_counter()
    for h, s, _ in probs:
        lapack.sygvd_chain(h, s)
    out_q.put((t0, time.perf_counter(), len(probs)))


def cpu_batch_throughput(sample=64, procs=None):
    """The reference's throughput protocol for the uneven batch (P processes x 1 thread, as its EigenBench sweeps,
    Sources/EigenBench/main.swift:464-497): `sample` problems of the 256-size draw (every (256/sample)-th in draw
    order; problem i built with seed 1000 + i), spread over P = nproc single-thread processes longest first (LPT by
    n^3), timed from the moment every process has built its inputs until the last one finishes.  Returns jobs/s and
    the sample's description.  Processes are started with `spawn` (never forked from a process that uses the GPU)."""
    import multiprocessing as mp

    sizes = batch_sizes(256, seed=3)
    step = max(1, 256 // sample)
    pick = list(range(0, 256, step))[:sample]
    procs = procs or (os.cpu_count() or 1)
    procs = max(1, min(procs, len(pick)))
    load = [0.0] * procs
    jobs = [[] for _ in range(procs)]
    for i in sorted(pick, key=lambda i: -sizes[i] ** 3):
        w = min(range(procs), key=lambda k: load[k])
        jobs[w].append((sizes[i], 1000 + i))
        load[w] += sizes[i] ** 3
    ctx = mp.get_context("spawn")
    barrier = ctx.Barrier(procs)
    out_q = ctx.Queue()
    ps = [ctx.Process(target=_cpu_batch_worker, args=(jobs[k], barrier, out_q)) for k in range(procs)]
    for p in ps:
        p.start()
    res = [out_q.get(timeout=1800) for _ in ps]
    for p in ps:
        p.join(timeout=60)
    wall = max(r[1] for r in res) - min(r[0] for r in res)
    return {"jobs_per_s": round(len(pick) / wall, 3), "processes": procs, "threads_per_process": 1,
            "problems": len(pick), "wall_s": round(wall, 2),
            "sample": f"{len(pick)} of the 256 uneven problems (every {step}th in draw order, sizes "
                      f"{min(sizes[i] for i in pick)}-{max(sizes[i] for i in pick)}), built with numpy seeds 1000 + i"}


def run_cpu_protocol(args):
    """The CPU baseline protocol on this host (no GPU): the reference's LAPACK chain for configurations 1-3 on one
    OpenBLAS thread and on all of them (median of 5 solves after one untimed solve, the reference's rule), and the
    uneven batch as P = nproc processes x 1 thread over all 256 problems (jobs/s).  One JSON line."""
    rank, _, _ = rank_info()
    if rank != 0:
        return
    from oracle import inputs, lapack

    nproc, model = host_cpu()
    t_all = lapack.get_threads()
    out = {"cpu_protocol": True, "host": {"nproc": nproc, "model": model, "openblas_threads_all": t_all},
           "rule": "median of 5 after 1 untimed solve", "configs": {}}
    cases = [("config1_standard_n412", "std", 412, 0), ("config2_generalized_n1204", "gen", 1204, 1),
             ("config3_generalized_n1788", "gen", 1788, 2)]
    for name, kind, n, seed in cases:
        if kind == "std":
            a, _ = inputs.standard(n, seed=seed)
            run = lambda: lapack.syevd_chain(a)  # noqa: E731
        else:
            h, s, _ = build_generalized(n, seed)
            run = lambda: lapack.sygvd_chain(h, s)  # noqa: E731
        rec = {}
        for label, threads in (("one_thread_ms", 1), ("all_cores_ms", t_all)):
            lapack.set_threads(threads)
            run()
            ts = []
            for _ in range(5):
                t0 = time.perf_counter()
                run()
                ts.append((time.perf_counter() - t0) * 1e3)
            rec[label] = round(statistics.median(ts), 3)
        lapack.set_threads(t_all)
        out["configs"][name] = rec
    out["configs"]["config4_batch_256"] = cpu_batch_throughput(sample=256)
    print(json.dumps(out), flush=True)


def run_reference(args):
    rank, _, world = rank_info()
    if rank != 0:
        return
    h, s, _ = build_generalized(args.n, args.seed)
    from oracle import lapack

    warm = max(3, min(args.warmup, 5))  # untimed solves, as many as the GPU arm's (at least 3), at most 5 (~3 s)
    for _ in range(warm):
        lapack.sygvd_chain(h, s)
    budget = 150.0
    ms, runs, threads = cpu_chain_time(h, s, budget, max(1, args.steps))
    line = {
        "impl": "reference", "metric": METRIC, "value": round(ms, 3), "unit": "ms", "n_gpus": world,
        "steps": runs, "warmup": warm, "ms_per_step": round(ms, 3), "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded generalized H, S; exact spectrum known)",
        "config": bench_config(args.n, args.seed),
        "details": {"path": "LAPACK dpotrf, dsygst, dsytrd, dstedc, dormtr, dtrsm (OpenBLAS 0.3.30 from scipy), "
                            "the reference's own call chain", "host_cpu": host_cpu()[1]},
        "cpu_baseline": {"value": round(ms, 3), "unit": "ms", "cores": host_cpu()[0], "threads": threads,
                         "kind": "port",
                         "sample": f"median of {runs} full solves on {threads} OpenBLAS threads (bounded to "
                                   f"~{int(budget)} s)"},
        "e2e": {"value": round(ms, 3), "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------------------------------------ GPU path

def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            pk = json.load(f)
        return float(pk.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


def load_traffic(n):
    """DRAM bytes per sytrd launch from the committed ncu summary (profiles/traffic.json): the kernel reads the matrix
    once and keeps it in shared memory, so traffic scales as n^2 when the capture was of another size; None if no
    capture exists."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        t = json.load(f)
    rec = t.get("sytrd")
    if not rec:
        return None
    return float(rec["bytes_per_launch"]) * (n / rec["n"]) ** 2 if rec.get("n") else None


def generalized_on_device(n, seed, dev):
    """The generalized construction (S = I + banded random G shifted to lambda_min >= 0.05, lam ~ U[-1, 0.5] Eh with a
    0.05 Eh gap at n/2, H = S^1/2 Q diag(lam) Q^T S^1/2) built on the GPU with torch's generator seeded `seed`: same
    distribution as the host builder (numpy's generator differs), used to make the 256 batch problems quickly.  The
    exact generalized spectrum is lam.  Input generation only, never timed."""
    import torch

    f64 = torch.float64
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    idx = torch.arange(n, device=dev, dtype=f64)
    dist = (idx[:, None] - idx[None, :]).abs()
    u = torch.rand((n, n), generator=g, device=dev, dtype=f64) * 2.0 - 1.0
    gm = 0.35 * torch.exp(-dist / 12.0) * torch.triu(u, 1)
    eye = torch.eye(n, device=dev, dtype=f64)
    s = eye + gm + gm.T
    lmin = float(torch.linalg.eigvalsh(s)[0])
    if lmin < 0.05:
        s += (0.05 - lmin) * eye
    lam = torch.sort(torch.rand(n, generator=g, device=dev, dtype=f64) * 1.5 - 1.0).values
    lam[n // 2:] += 0.05
    q, r = torch.linalg.qr(torch.randn((n, n), generator=g, device=dev, dtype=f64))
    q = q * torch.sign(torch.diagonal(r))[None, :]
    ws, vs = torch.linalg.eigh(s)
    shalf = (vs * torch.sqrt(ws)[None, :]) @ vs.T
    shalf = 0.5 * (shalf + shalf.T)
    h = shalf @ ((q * lam[None, :]) @ q.T) @ shalf
    h = 0.5 * (h + h.T)
    return h.contiguous(), s.contiguous(), lam


def accuracy_on_device(H, S, lam, C, w, C_ref):
    """Errors of (w, C) for H C = S C diag(w) (torch float64 on the device, C column vectors): eigenvalues against
    the exact spectrum lam, backward error ||HC - SC diag(w)||_F / (||H||_F n eps), S-orthogonality max|C^T S C - I|,
    and the aufbau density (2 electrons in the lower half) against C_ref's.  Measurement only (torch matmuls)."""
    import torch

    n = H.shape[0]
    eps = 2.0 ** -53
    r = H @ C - (S @ C) * w[None, :]
    bwd = float(torch.linalg.norm(r) / (torch.linalg.norm(H) * n * eps))
    orth = float((C.T @ S @ C - torch.eye(n, dtype=C.dtype, device=C.device)).abs().max())
    m = n // 2
    p = 2.0 * C[:, :m] @ C[:, :m].T
    p_ref = 2.0 * C_ref[:, :m] @ C_ref[:, :m].T
    return {"eigenvalue_error_vs_exact": float((w - lam).abs().max()), "backward_error": bwd,
            "s_orthogonality": orth, "density_error_vs_fp64_gpu": float((p - p_ref).abs().max())}


def oracle_errors(dev, W, C, oracle):
    """Eigenvalue and aufbau-density errors of (W, C) (device) against the CPU LAPACK chain's (w, C)."""
    import numpy as np
    import torch

    if oracle is None:
        return {}
    w_or, c_or = oracle
    m = C.shape[0] // 2
    Co = torch.from_numpy(np.ascontiguousarray(c_or[:, :m])).to(dev)
    return {"eigenvalue_error_vs_oracle": float((W.cpu() - torch.from_numpy(w_or)).abs().max()),
            "density_error_vs_oracle": float((2.0 * C[:, :m] @ C[:, :m].T - 2.0 * Co @ Co.T).abs().max())}


def run_mixed_section(args, dev, stream, H0, S0, lam_t, C64, flush, oracle=None):
    """The same n = 1788 solve with precision 32: FP32 congruence, resident sytrd, ormtr and back-transform (FP64
    Cholesky and tridiagonal eigensolve), then FP64 refinement (two Ogita-Aishima steps) on the FP64 pair.  Timed like
    the FP64 path; accuracy against the exact spectrum and the FP64 GPU result."""
    import torch

    import xtbeig

    n = H0.shape[0]
    H, S = torch.empty_like(H0), torch.empty_like(S0)
    W = torch.empty(n, dtype=torch.float64, device=dev)

    def solve():
        H.copy_(H0)
        S.copy_(S0)
        info = xtbeig.dsygvd_device(n, H.data_ptr(), n, S.data_ptr(), n, W.data_ptr(), stream.cuda_stream)
        if info != 0:
            raise RuntimeError(f"mixed xtb_dsygvd_device info={info}: {xtbeig.last_error()}")

    xtbeig.set_option("precision", 32)
    try:
        for _ in range(3):
            solve()
        torch.cuda.synchronize(dev)
        acc = accuracy_on_device(H0, S0, lam_t, H.T, W, C64)
        acc.update(oracle_errors(dev, W, H.T, oracle))
        xtbeig.set_option("stage_timing", 1)
        flush.zero_()
        solve()
        stages = xtbeig.stage_times()
        xtbeig.set_option("stage_timing", 0)
        solve()  # untimed: the stage-timed solve ran eagerly, so this one may (re)capture the solve's graph
        K = max(1, args.steps // 2)
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
        torch.cuda.nvtx.range_push("mixed_timed")
        for i in range(K):
            flush.zero_()
            ev[i][0].record(stream)
            solve()
            ev[i][1].record(stream)
        torch.cuda.synchronize(dev)
        torch.cuda.nvtx.range_pop()
        ms = sum(a.elapsed_time(b) for a, b in ev) / K
    finally:
        xtbeig.set_option("precision", 64)
    out = {"ms": round(ms, 4), "steps": K, "warmup": 3, "refine_iters": xtbeig.get_option("refine_iters"),
           "stages_ms": {k: round(v, 4) for k, v in stages}}
    out.update(acc)
    return out


def run_variant_section(args, dev, stream, H0, S0, lam_t, flush, options, steps=3, C64=None, oracle=None):
    """The n = 1788 solve under other library options (e.g. the two-stage reduction): mean ms over `steps` timed
    solves after 3 warm-ups, stage times of one untimed solve, eigenvalue error against the exact spectrum; with C64
    (the FP64 GPU solve's C) the backward error, S-orthogonality and density error (accuracy_on_device), and with
    `oracle` (the CPU LAPACK chain's (w, C), computed by the cpu_baseline leg) the eigenvalue and density errors
    against it.  A solve that returns a nonzero info is reported, not raised."""
    import torch

    import xtbeig

    n = H0.shape[0]
    H, S = torch.empty_like(H0), torch.empty_like(S0)
    W = torch.empty(n, dtype=torch.float64, device=dev)
    old = {k: xtbeig.get_option(k) for k in options}

    def solve():
        H.copy_(H0)
        S.copy_(S0)
        info = xtbeig.dsygvd_device(n, H.data_ptr(), n, S.data_ptr(), n, W.data_ptr(), stream.cuda_stream)
        if info != 0:
            raise RuntimeError(f"xtb_dsygvd_device info={info}: {xtbeig.last_error()}")

    acc = {}
    try:
        for k, v in options.items():
            xtbeig.set_option(k, v)
        try:
            for _ in range(3):
                solve()
        except RuntimeError as e:
            return {"options": options, "failed": str(e)}
        torch.cuda.synchronize(dev)
        err = float((W - lam_t).abs().max())
        if C64 is not None:
            acc = accuracy_on_device(H0, S0, lam_t, H.T, W, C64)
        acc.update(oracle_errors(dev, W, H.T, oracle))
        xtbeig.set_option("stage_timing", 1)
        solve()
        stages = xtbeig.stage_times()
        xtbeig.set_option("stage_timing", 0)
        solve()  # untimed: the stage-timed solve ran eagerly, so this one may (re)capture the solve's graph
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        for i in range(steps):
            flush.zero_()
            ev[i][0].record(stream)
            solve()
            ev[i][1].record(stream)
        torch.cuda.synchronize(dev)
        ms = sum(a.elapsed_time(b) for a, b in ev) / steps
    finally:
        for k, v in old.items():
            xtbeig.set_option(k, v)
    out = {"options": options, "ms": round(ms, 4), "steps": steps, "warmup": 3, "eigenvalue_error_vs_exact": err,
           "stages_ms": {k: round(v, 4) for k, v in stages}}
    out.update(acc)
    return out


def run_cycle_section(args, dev, stream, H0, S0, lam_t, flush, precision, steps=5):
    """The per-SCC-cycle solve: S factored once (xtb_dsygvd_factor_device, untimed), then `steps` timed solves of the
    same H with that factorization (xtb_dsygvd_factored_device: congruence, reduction, tridiagonal eigensolve,
    back-transformations and, at precision 32, the refinement)."""
    import torch

    import xtbeig

    n = H0.shape[0]
    U = S0.clone()
    X = torch.empty_like(S0)
    H = torch.empty_like(H0)
    W = torch.empty(n, dtype=torch.float64, device=dev)
    prec0 = xtbeig.get_option("precision")
    xtbeig.set_option("precision", precision)
    try:
        if xtbeig.dsygvd_factor_device(n, U.data_ptr(), n, X.data_ptr(), n, stream.cuda_stream) != 0:
            raise RuntimeError(f"xtb_dsygvd_factor_device: {xtbeig.last_error()}")

        def solve():
            H.copy_(H0)
            info = xtbeig.dsygvd_factored_device(n, H.data_ptr(), n, U.data_ptr(), n, X.data_ptr(), n, W.data_ptr(),
                                                 stream.cuda_stream)
            if info != 0:
                raise RuntimeError(f"xtb_dsygvd_factored_device info={info}: {xtbeig.last_error()}")

        for _ in range(3):
            solve()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        for i in range(steps):
            flush.zero_()
            ev[i][0].record(stream)
            solve()
            ev[i][1].record(stream)
        torch.cuda.synchronize(dev)
        ms = sum(a.elapsed_time(b) for a, b in ev) / steps
        err = float((W - lam_t).abs().max())
    finally:
        xtbeig.set_option("precision", prec0)
    return {"ms": round(ms, 4), "steps": steps, "warmup": 3, "eigenvalue_error_vs_exact": err}


def run_reuse_section(args, dev, stream, H0, S0, flush, eps=1e-4, steps=5):
    """The eigenvector-reuse cycle (the reference's refine.f90 method_oa_from): the converged C of H0 is refined against
    a perturbed H1 = H0 + eps sym(R) (R seeded N(0, 1); late SCC cycles change H by little, early ones by more) with
    xtb_dsygvd_refine_device, 1 and 2 Ogita-Aishima steps.  Reported: ms per refinement (the copy of C0 into the work
    buffer is outside the timed region), and its errors against a full FP64 solve of (H1, S0): eigenvalues and the
    aufbau density."""
    import torch

    import xtbeig

    n = H0.shape[0]
    g = torch.Generator(device=dev)
    g.manual_seed(4242)
    r = torch.randn((n, n), generator=g, device=dev, dtype=torch.float64)
    H1 = (H0 + 0.5 * eps * (r + r.T)).contiguous()
    H, S = torch.empty_like(H0), torch.empty_like(S0)
    W0 = torch.empty(n, dtype=torch.float64, device=dev)
    W1 = torch.empty(n, dtype=torch.float64, device=dev)

    def full(hsrc, w):
        H.copy_(hsrc)
        S.copy_(S0)
        info = xtbeig.dsygvd_device(n, H.data_ptr(), n, S.data_ptr(), n, w.data_ptr(), stream.cuda_stream)
        if info != 0:
            raise RuntimeError(f"xtb_dsygvd_device info={info}: {xtbeig.last_error()}")
        torch.cuda.synchronize(dev)
        return H.clone()  # column-major C in the row-major view: C^T

    C0t = full(H0, W0)
    C1t = full(H1, W1)
    m = n // 2
    P1 = 2.0 * C1t[:m].T @ C1t[:m]
    Ct = torch.empty_like(C0t)
    W = torch.empty(n, dtype=torch.float64, device=dev)
    out = {"eps": eps, "n": n, "perturbation": "H1 = H0 + eps (R + R^T)/2, R ~ N(0, 1) seeded 4242",
           "start_eigenvalue_change": float((W1 - W0).abs().max())}
    for iters in (1, 2):
        def refine():
            info = xtbeig.dsygvd_refine_device(n, H1.data_ptr(), n, S0.data_ptr(), n, Ct.data_ptr(), n, W.data_ptr(),
                                               iters, stream.cuda_stream)
            if info != 0:
                raise RuntimeError(f"xtb_dsygvd_refine_device info={info}: {xtbeig.last_error()}")

        for _ in range(3):
            Ct.copy_(C0t)
            refine()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        for i in range(steps):
            Ct.copy_(C0t)
            flush.zero_()
            ev[i][0].record(stream)
            refine()
            ev[i][1].record(stream)
        torch.cuda.synchronize(dev)
        ms = sum(a.elapsed_time(b) for a, b in ev) / steps
        P = 2.0 * Ct[:m].T @ Ct[:m]
        out[f"iters_{iters}"] = {"ms": round(ms, 4), "steps": steps, "warmup": 3,
                                 "eigenvalue_error_vs_fp64_solve": float((W - W1).abs().max()),
                                 "density_error_vs_fp64_solve": float((P - P1).abs().max())}
    return out


def run_adjoint_section(args, dev):
    """The differentiation workload: `count` generalized problems at n = 588 (problem i built on the device with seed
    4000 + i), Fermi occupations at T = 300 K with mu at mid-gap, W symmetric standard normal; dL/dH and dL/dS of
    L = sum(W o P) through xtb_dsygvd_density_adjoint_batched (host arrays: each problem's solve, eigenvectors and
    adjoint on the GPU, nothing stored), timed end to end in FP64 and in mixed precision."""
    import numpy as np
    import torch

    import xtbeig
    from oracle import fermi

    count, n = args.adjoint_count, 588
    hs, ss, mus, wbs = [], [], [], []
    rng = np.random.default_rng(4)
    for i in range(count):
        h, s, lam = generalized_on_device(n, 4000 + i, dev)
        hs.append(np.asfortranarray(h.cpu().numpy()))
        ss.append(np.asfortranarray(s.cpu().numpy()))
        lam = lam.cpu().numpy()
        mus.append(0.5 * (lam[n // 2 - 1] + lam[n // 2]))
        w = rng.standard_normal((n, n))
        wbs.append(np.asfortranarray(w + w.T))
    kts = [fermi.kt_of(300.0)] * count
    out = {"count": count, "n": n, "temperature_K": 300.0}
    prec0 = xtbeig.get_option("precision")
    try:
        for name, prec in (("fp64", 64), ("mixed", 32)):
            if prec == 32 and args.no_mixed:
                continue
            xtbeig.set_option("precision", prec)
            xtbeig.density_adjoint_batched(hs, ss, kts, mus, wbs)  # warm-up: every worker's context and buffers
            t0 = time.perf_counter()
            _, _, info = xtbeig.density_adjoint_batched(hs, ss, kts, mus, wbs)
            dt = time.perf_counter() - t0
            if np.any(info != 0):
                raise RuntimeError(f"adjoint batch info {info}")
            out[name] = {"ms_per_batch": round(dt * 1e3, 2), "problems_per_s": round(count / dt, 2)}
    finally:
        xtbeig.set_option("precision", prec0)
    if "mixed" in out:
        out["mixed_speedup_vs_fp64"] = round(out["fp64"]["ms_per_batch"] / out["mixed"]["ms_per_batch"], 3)
    out["note"] = "end to end through the C ABI from host arrays (H, S, W in; dL/dH, dL/dS out); accuracy is tested"
    return out


def batch_sizes(count, seed=3, lo=124, hi=1788):
    """Sizes of the uneven batch: integers uniform in [lo, hi] from numpy's default_rng(seed)."""
    import numpy as np

    return [int(x) for x in np.random.default_rng(seed).integers(lo, hi + 1, count)]


def run_batch_section(args, dev, stream, rank=0, world=1):
    """The uneven batch: `count` generalized problems, sizes U[124, 1788] (seed 3), problem i built with seed
    1000 + i.  Device-resident batches through xtb_dsygvd_batched_device (restore of H, S inside each timed step),
    the same problems solved one at a time through xtb_dsygvd_device (per-size times), and one end-to-end batch
    through xtb_dsygvd_batched from pinned host arrays.  With N ranks the batch is sharded: every rank builds and solves
    only its own problems (xtb_batch_partition, longest first on the cost model of n; no exchange), and the batch
    time is the maximum over ranks (one-at-a-time times are measured at N = 1 only)."""
    import ctypes

    import numpy as np
    import torch

    import shard
    import xtbeig

    count = args.batch_count
    all_sizes = batch_sizes(count, seed=3)
    mine = shard.my_problems(all_sizes, rank, world) if world > 1 else list(range(count))

    def max_over_ranks(x):
        if world == 1:
            return x
        import torch.distributed as dist

        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    sizes = [all_sizes[i] for i in mine]
    t0 = time.perf_counter()
    H0, S0, LAM = [], [], []
    for i, n in zip(mine, sizes):
        h, s, lam = generalized_on_device(n, 1000 + i, dev)
        H0.append(h)
        S0.append(s)
        LAM.append(lam)
    torch.cuda.synchronize(dev)
    gen_s = time.perf_counter() - t0
    H = [torch.empty_like(x) for x in H0]
    S = [torch.empty_like(x) for x in S0]
    W = [torch.empty(n, dtype=torch.float64, device=dev) for n in sizes]
    hp, sp, wp = [x.data_ptr() for x in H], [x.data_ptr() for x in S], [x.data_ptr() for x in W]

    nloc = len(sizes)

    def batch_step():
        for i in range(nloc):
            H[i].copy_(H0[i])
            S[i].copy_(S0[i])
        info, r = xtbeig.dsygvd_batched_device(sizes, hp, sizes, sp, sizes, wp, stream.cuda_stream)
        if r != 0:
            raise RuntimeError(f"xtb_dsygvd_batched_device returned {r}: {xtbeig.last_error()}")

    workers = xtbeig.get_option("batch_workers")
    for _ in range(3):  # eager, captured, replayed
        batch_step()
    torch.cuda.synchronize(dev)
    steps = max(1, args.batch_steps)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    launches0 = xtbeig.launch_count()
    torch.cuda.nvtx.range_push("batch_timed")
    for k in range(steps):
        ev[k][0].record(stream)
        batch_step()
        ev[k][1].record(stream)
    torch.cuda.synchronize(dev)
    torch.cuda.nvtx.range_pop()
    launches = xtbeig.launch_count() - launches0
    ms_batch = max_over_ranks(statistics.mean(a.elapsed_time(b) for a, b in ev))
    eig_err = max_over_ranks(max(float((W[i] - LAM[i]).abs().max()) for i in range(nloc)))

    # The same batch in mixed precision (FP32 reduction chain + FP64 refinement).
    mixed = None
    if not args.no_mixed:
        prec0 = xtbeig.get_option("precision")
        xtbeig.set_option("precision", 32)
        try:
            for _ in range(3):
                batch_step()
            torch.cuda.synchronize(dev)
            evm = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
            for k in range(steps):
                evm[k][0].record(stream)
                batch_step()
                evm[k][1].record(stream)
            torch.cuda.synchronize(dev)
            ms_m = max_over_ranks(statistics.mean(a.elapsed_time(b) for a, b in evm))
            err_m = max_over_ranks(max(float((W[i] - LAM[i]).abs().max()) for i in range(nloc)))
        finally:
            xtbeig.set_option("precision", prec0)
        mixed = {"solves_per_s": round(count / (ms_m * 1e-3), 2), "ms_per_batch": round(ms_m, 2), "steps": steps,
                 "warmup": 3, "speedup_vs_fp64_batch": round(ms_batch / ms_m, 3),
                 "eigenvalue_error_vs_exact_max": err_m}

    # One at a time: each problem alone on the caller's stream (eager, captured, then the timed replay).
    per = []
    for i, n in enumerate(sizes if world == 1 else []):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        for rep in range(3):
            H[i].copy_(H0[i])
            S[i].copy_(S0[i])
            if rep == 2:
                e0.record(stream)
            info = xtbeig.dsygvd_device(n, hp[i], n, sp[i], n, wp[i], stream.cuda_stream)
            if info != 0:
                raise RuntimeError(f"xtb_dsygvd_device info={info}: {xtbeig.last_error()}")
        e1.record(stream)
        torch.cuda.synchronize(dev)
        per.append(e0.elapsed_time(e1))
    one_ms = sum(per) if per else None
    bins = {}
    for lo, hi in ((124, 500), (500, 900), (900, 1300), (1300, 1789)):
        sel = [t for n, t in zip(sizes, per) if lo <= n < hi]
        if sel:
            bins[f"{lo}-{hi - 1}"] = {"count": len(sel), "mean_ms_alone": round(statistics.mean(sel), 3)}

    # End to end through the host C ABI: pinned host H, S in, C, U, w back.
    L = xtbeig.lib()
    hh = [torch.empty((n, n), dtype=torch.float64, pin_memory=True) for n in sizes]
    sh = [torch.empty((n, n), dtype=torch.float64, pin_memory=True) for n in sizes]
    wh = [torch.empty(n, dtype=torch.float64, pin_memory=True) for n in sizes]
    ns = np.array(sizes, np.int32)
    ap = (ctypes.c_void_p * nloc)(*[x.data_ptr() for x in hh])
    bp = (ctypes.c_void_p * nloc)(*[x.data_ptr() for x in sh])
    wq = (ctypes.c_void_p * nloc)(*[x.data_ptr() for x in wh])
    infos = np.zeros(nloc, np.int32)
    e2e = []
    for rep in range(2):
        for i in range(nloc):
            hh[i].copy_(H0[i])
            sh[i].copy_(S0[i])
        t1 = time.perf_counter()
        r = L.xtb_dsygvd_batched(nloc, xtbeig._p(ns), ap, xtbeig._p(ns), bp, xtbeig._p(ns), wq, xtbeig._p(infos))
        dt = max_over_ranks(time.perf_counter() - t1)
        if r != 0:
            raise RuntimeError(f"xtb_dsygvd_batched returned {r}: {xtbeig.last_error()}")
        if rep == 1:
            e2e.append(dt)
    elems = sum(all_sizes[i] ** 2 for i in range(count))
    return {
        "count": count, "sizes": "uniform integers in [124, 1788], seed 3; problem i built with seed 1000 + i",
        "sharding": (f"{world} ranks, each solving its own problems (xtb_batch_partition); times are the maximum over "
                     "ranks" if world > 1 else "one GPU"),
        "workers": workers, "batch_grid": xtbeig.get_option("batch_grid"),
        "solves_per_s": round(count / (ms_batch * 1e-3), 2), "ms_per_batch": round(ms_batch, 2),
        "steps": steps, "warmup": 3, "gpu_launches_per_batch": int(launches // steps),
        "one_at_a_time_solves_per_s": round(count / (one_ms * 1e-3), 2) if one_ms else None,
        "one_at_a_time_ms": round(one_ms, 2) if one_ms else None,
        "speedup_vs_one_at_a_time": round(one_ms / ms_batch, 3) if one_ms else None, "per_size_ms_alone": bins,
        "eigenvalue_error_vs_exact_max": eig_err,
        "mixed": mixed,
        "e2e": {"solves_per_s": round(count / e2e[0], 2), "ms_per_batch": round(e2e[0] * 1e3, 2),
                "h2d_bytes_per_batch": 2 * sum(triangle_bytes(m) for m in all_sizes[:count]),
                "d2h_bytes_per_batch": (elems + sum(all_sizes[:count])) * 8
                + sum(triangle_bytes(m) for m in all_sizes[:count])},
        "l2": "not flushed: the batch's matrices (~%.1f GB) exceed L2" % (4 * elems * 8 / 1e9),
        "input_generation_s": round(gen_s, 1),
        "input_builder": "torch on the device (generator seeded per problem), outside every timed region",
    }


def run_ours(args):
    import numpy as np
    import torch
    import torch.distributed as dist

    import xtbeig

    rank, local_rank, world = rank_info()
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    torch.cuda.set_device(local_rank)
    xtbeig.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    n = args.n
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    if args.hs_bin:
        import hsbin

        dump = hsbin.read_hs_bin(args.hs_bin)
        n = args.n = dump["n"]
        # symmetric: row-major == column-major
        H0 = torch.from_numpy(np.ascontiguousarray(dump["h"])).to(dev)
        S0 = torch.from_numpy(np.ascontiguousarray(dump["s"])).to(dev)
        lam_t = None  # no exact spectrum: errors are reported against the FP64 GPU solve
    else:
        # The same host-built bytes as the CPU arm (symmetric: row-major == column-major on the device).
        h_np, s_np, lam_np = build_generalized(n, args.seed)
        H0 = torch.from_numpy(np.ascontiguousarray(h_np)).to(dev)
        S0 = torch.from_numpy(np.ascontiguousarray(s_np)).to(dev)
        lam_t = torch.from_numpy(lam_np).to(dev)
    h_np, s_np = H0.cpu().numpy(), S0.cpu().numpy()
    H = torch.empty_like(H0)
    S = torch.empty_like(S0)
    W = torch.empty(n, dtype=torch.float64, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def solve():
        H.copy_(H0)
        S.copy_(S0)
        info = xtbeig.dsygvd_device(n, H.data_ptr(), n, S.data_ptr(), n, W.data_ptr(), stream.cuda_stream)
        if info != 0:
            raise RuntimeError(f"xtb_dsygvd_device info={info}: {xtbeig.last_error()}")

    # Autotuning (outside every timed region): the fastest plan of each precision for this size.
    plans = None
    if not args.no_autotune:
        t0 = time.perf_counter()
        plans = {"fp64": xtbeig.autotune(n, 64, stream.cuda_stream)}
        if not args.no_mixed:
            plans["mixed"] = xtbeig.autotune(n, 32, stream.cuda_stream)
        plans["tuning_s"] = round(time.perf_counter() - t0, 2)
        xtbeig.set_option("autotune", 1)

    for _ in range(max(3, args.warmup)):
        solve()
    torch.cuda.synchronize(dev)
    eig_reference = "exact spectrum of the construction"
    if lam_t is None:
        lam_t = W.clone()
        eig_reference = "FP64 GPU solve (the dump has no exact spectrum)"
    lam = lam_t.cpu().numpy()
    # accuracy of the measured configuration (outside the timed region)
    w = W.cpu().numpy()
    eig_err = float(np.max(np.abs(w - lam)))
    C64 = H.T.contiguous()
    acc64 = accuracy_on_device(H0, S0, lam_t, C64, W.clone(), C64)
    # The checker for the accuracy fields: the reference's LAPACK chain on the same bytes (the cpu_baseline leg's
    # computation; one GPU only, never timed here).
    oracle = None
    if world == 1 and not args.no_cpu_baseline and not args.hs_bin:
        oracle = cpu_reference_solution(h_np, s_np)
        acc64.update(oracle_errors(dev, W, C64, oracle))

    # Stage times of one untimed solve (CUDA events at stage boundaries inside the library).
    xtbeig.set_option("stage_timing", 1)
    flush.zero_()
    solve()
    stages = xtbeig.stage_times()
    xtbeig.set_option("stage_timing", 0)
    solve()  # untimed: the stage-timed solve ran eagerly, so this one may (re)capture the solve's graph
    torch.cuda.synchronize(dev)

    # Timed region.
    gpu_uuid = str(torch.cuda.get_device_properties(dev).uuid)
    sampler = ClockSampler(("GPU-" + gpu_uuid) if not gpu_uuid.startswith("GPU-") else gpu_uuid)
    K = args.steps
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    launches0 = xtbeig.launch_count()
    sampler.start()
    time.sleep(0.3)
    t_wall0 = time.perf_counter()
    torch.cuda.nvtx.range_push("fp64_timed")
    for i in range(K):
        flush.zero_()
        ev[i][0].record(stream)
        solve()
        ev[i][1].record(stream)
    torch.cuda.synchronize(dev)
    torch.cuda.nvtx.range_pop()
    t_wall = time.perf_counter() - t_wall0
    if world > 1:
        dist.barrier()
    clocks = sampler.stop()
    launches = xtbeig.launch_count() - launches0
    per = [a.elapsed_time(b) for a, b in ev]
    ms_step = sum(per) / K
    t = torch.tensor([ms_step], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_step_max = float(t.item())

    # End to end through the C ABI with pinned host buffers.
    import ctypes

    L = xtbeig.lib()
    hp = torch.empty((n, n), dtype=torch.float64, pin_memory=True).numpy()
    sp = torch.empty((n, n), dtype=torch.float64, pin_memory=True).numpy()
    wp = torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()
    hf, sf = np.ascontiguousarray(h_np), np.ascontiguousarray(s_np)
    info = ctypes.c_int(0)
    one = ctypes.c_int(1)
    e2e = []
    for i in range(args.e2e_steps + 2):
        np.copyto(hp, hf)
        np.copyto(sp, sf)
        t0 = time.perf_counter()
        L.xtb_dsygvd_gpu(ctypes.byref(one), b"V", b"U", ctypes.byref(ctypes.c_int(n)), xtbeig._p(hp),
                         ctypes.byref(ctypes.c_int(n)), xtbeig._p(sp), ctypes.byref(ctypes.c_int(n)), xtbeig._p(wp),
                         None, ctypes.byref(one), None, ctypes.byref(one), ctypes.byref(info))
        dt = (time.perf_counter() - t0) * 1e3
        if info.value != 0:
            raise RuntimeError(f"xtb_dsygvd_gpu info={info.value}: {xtbeig.last_error()}")
        if i >= 2:
            e2e.append(dt)
    e2e_ms = statistics.median(e2e)
    te = torch.tensor([e2e_ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e_ms = float(te.item())

    mixed = run_mixed_section(args, dev, stream, H0, S0, lam_t, C64, flush, oracle) if not args.no_mixed else None
    if mixed:
        mixed["speedup_vs_fp64"] = round(ms_step_max / mixed["ms"], 3)
    cycle = {"fp64": run_cycle_section(args, dev, stream, H0, S0, lam_t, flush, 64)}
    cycle["eigenvector_reuse"] = {f"eps_{eps:.0e}": run_reuse_section(args, dev, stream, H0, S0, flush, eps=eps)
                                  for eps in (1e-6, 1e-5, 1e-4)}
    if not args.no_mixed:
        cycle["mixed"] = run_cycle_section(args, dev, stream, H0, S0, lam_t, flush, 32)
        cycle["mixed_speedup_vs_fp64"] = round(cycle["fp64"]["ms"] / cycle["mixed"]["ms"], 3)
    two_stage = None
    if not args.no_two_stage:
        # FP64 at the band widths its panel fits in shared memory; the FP32 chain (then FP64 refinement) with its GEMMs
        # on each tensor-core engine at b = 32, 64, 128: the accuracy table of the mixed two-stage design.
        two_stage = {"fp64": {f"b{b}": run_variant_section(args, dev, stream, H0, S0, lam_t, flush,
                                                           {"autotune": 0, "reduction": 2, "band_width": b},
                                                           C64=C64, oracle=oracle)
                              for b in (32, 64)}}
        if not args.no_mixed:
            engines = {"tf32": 1, "3xtf32": 3, "bf16": 11, "3xbf16": 13}
            two_stage["mixed"] = {
                f"{name}_b{b}": run_variant_section(args, dev, stream, H0, S0, lam_t, flush,
                                                    {"autotune": 0, "reduction": 2, "band_width": b, "precision": 32,
                                                     "mixed_gemm": eng}, C64=C64, oracle=oracle)
                for name, eng in engines.items() for b in (32, 64, 128)}
    batch = run_batch_section(args, dev, stream, rank, world) if args.batch_count > 0 else None
    adjoint = run_adjoint_section(args, dev) if args.adjoint_count > 0 else None

    if rank == 0:
        peak, peak_kind = load_peaks()
        t_sytrd = dict(stages).get("sytrd")
        alg_bytes = 4.0 * n ** 3 / 3.0
        achieved = alg_bytes / (t_sytrd * 1e-3) / 1e9 if t_sytrd else None
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            ms_cpu, runs, threads = cpu_chain_time(h_np, s_np, args.cpu_budget_s, 50)
            ms_one, runs_one = cpu_one_thread_time(h_np, s_np)
            nproc, model = host_cpu()
            cpu = {"value": round(ms_cpu, 3), "unit": "ms", "cores": nproc, "threads": threads, "kind": "port",
                   "sample": f"median of {runs} full n={n} solves of the LAPACK chain (OpenBLAS) on {threads} "
                             f"threads, <= {args.cpu_budget_s:.0f} s",
                   "one_thread": {"ms": round(ms_one, 3), "runs": runs_one,
                                  "sample": f"median of {runs_one} full n={n} solves on 1 OpenBLAS thread"},
                   "host_cpu": model}
            if args.batch_count > 0 and args.cpu_batch_sample > 0:
                cpu["batch_p_x_1"] = cpu_batch_throughput(args.cpu_batch_sample)
        total_stage = sum(v for _, v in stages) or 1.0
        line = {
            "metric": METRIC, "value": round(ms_step_max / world, 4), "unit": "ms", "n_gpus": world, "steps": K,
            "warmup": max(3, args.warmup), "ms_per_step": round(ms_step_max, 4), "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded generalized H, S; exact spectrum known)",
            "config": ({"workload": f"generalized eigensolve of {os.path.basename(args.hs_bin)} n={n}, all "
                                    "eigenpairs, FP64", "l2": "flushed (256 MB write) before every timed step"}
                       if args.hs_bin else bench_config(n, args.seed)),
            "details": {"eigenvalue_reference": eig_reference,
                       "path": "potrf, trtri, X^T H X, resident sytrd, D&C stedc, WY ormtr, X C' (all CUDA)",
                       "multi_gpu": ("one GPU" if world == 1 else f"{world} independent replicas of the solve (a single "
                                     "solve does not shard); value = max-over-ranks ms per step / N"),
                       "fp64_gemm_engine": ("int8 Ozaki splitting on tcgen05 for GEMMs >= 512^3 (exact int32 slice "
                                            "products, one FP64 rounding; FP64 accuracy), DMMA below"
                                            if (plans["fp64"]["dgemm"] if plans else
                                                xtbeig.get_option("dgemm_engine")) else "FP64 DMMA"),
                       "l2": "flushed (256 MB write) before every timed step", "parallelism": f"replicas x{world}",
                       "eigenvalue_error_vs_exact": eig_err, "wall_s_timed_region": round(t_wall, 3)},
            "roofline": {"bound": "hbm", "kernel": "sytrd_resident_kernel",
                         "achieved": round(achieved, 1) if achieved else None, "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4) if achieved else None, "traffic": load_traffic(n),
                         "peak_kind": f"{peak_kind} copy bandwidth",
                         "algorithmic_bytes_per_launch": alg_bytes, "launch_ms": t_sytrd},
            "stages_ms": {k: round(v, 4) for k, v in stages},
            "stage_share": {k: round(v / total_stage, 3) for k, v in stages},
            "cpu_baseline": cpu,
            "e2e": {"value": round(e2e_ms / world, 4), "unit": "ms",
                    "h2d_bytes_per_step": 2 * triangle_bytes(n),
                    "d2h_bytes_per_step": (n * n + n) * 8 + triangle_bytes(n) + 16,
                    "transfers": "H and S up, C (whole), U and w down; H, S and U as their upper triangles",
                    "per_replica_ms": round(e2e_ms, 4)},
            "gpu_launches": int(launches),
            "clocks": clocks,
            "fp64_accuracy": acc64,
            "plans": plans,
            "scc_cycle": cycle,
            "mixed": mixed,
            "two_stage": two_stage,
            "batch": batch,
            "adjoint": adjoint,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def main():
    args = parse()
    if args.cpu_protocol:
        run_cpu_protocol(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
