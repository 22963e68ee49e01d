"""Benchmark: seconds per 128-alpha SpecAnn solve on a Barabasi-Albert graph (default n = 2^20, m = 20,
J = -A, fp32 couplings, int32 columns), the paper's SpecAnn run (sqrt schedule, diagonal predictor,
eigsh tolerance 1e-6, batched local search), plus the fused SpMV's HBM bandwidth.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--log2n 20] [--m 20]

A step is one full solve (prelude, 128 eigensolves, rounding, deduplication, batched local search,
best candidate). `value` is timed with the CSR already in HBM (SpectralAnnealing.solve_device);
`e2e` is the same metric through SpectralAnnealing.solve(J) with a host SciPy CSR, so every step
includes the host-to-device copy of the matrix and the device-to-host copy of the best spins.
Under torchrun each rank solves its own seed of the same graph (independent replicas, no collective
on the data path); `value` is the max-over-ranks step time divided by the number of solves.

--impl reference times the CPU reference pipeline (the oracle port: SciPy ARPACK eigsh + NumPy local
search) on a bounded sample of the same workload and extrapolates to a full 128-alpha solve.
"""
import argparse
import json
import os
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "s per 128-alpha SpecAnn solve (BA m=20, sqrt schedule, FP32 + FP64 Ritz); SpMV HBM GB/s"
UNIT = "s/solve"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--log2n", type=int, default=20)
    ap.add_argument("--m", type=int, default=20)
    ap.add_argument("--num-alphas", type=int, default=128)
    ap.add_argument("--precision", type=int, default=32)
    ap.add_argument("--e2e-steps", type=int, default=None)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-sample-alphas", type=int, default=2)
    ap.add_argument("--ref-candidates", type=int, default=128,
                    help="reference arm: distinct candidates of a full solve (the GPU run's count)")
    ap.add_argument("--ref-ls-passes", type=int, default=89,
                    help="reference arm: local-search passes of a full solve (89: the count of the default "
                         "workload's solve, seed 42, whose local search is bit-exact with the CPU one)")
    ap.add_argument("--spmv-reps", type=int, default=20)
    ap.add_argument("--batch-count", type=int, default=64,
                    help="--workload batch: instances of the ragged batch (64: the workload; fewer for profiling)")
    ap.add_argument("--workload", default="metric", choices=["metric", "batch", "precision", "grad"],
                    help="metric: the headline solve (default); batch: the ragged batched workload "
                         "(64 instances x 4 seeds x 128 alphas, one launch); precision: FP32 + FP64 Ritz vs "
                         "all-FP64 on BA(2^16); grad: the differentiation workload on BA(2^18)")
    ap.add_argument("--scale-precisions", default="32,64", help="--scale-run: precisions to run, in order")
    ap.add_argument("--scale-log2n", type=int, default=25,
                    help="the default line's scale block: log2 n of its BA graph (0: no scale block)")
    ap.add_argument("--scale-maxiter", type=int, default=1000,
                    help="eigsh_maxiter of the scale solves (the reference's default is 1000)")
    ap.add_argument("--scale-run", action="store_true",
                    help="one timed FP32 solve and one timed plain-FP64 solve of the graph, with the energy gap")
    ap.add_argument("--spmv-layout", choices=["auto", "panel", "split", "worklist"], default="auto",
                    help="operator layout of --spmv-only (auto: the solver's choice)")
    ap.add_argument("--spmv-only", action="store_true",
                    help="time only the standalone fused SpMV on the resident matrix (profiling runs)")
    return ap.parse_args()


def traffic_ratio():
    """DRAM bytes / algorithmic bytes of one captured alpha_kernel launch (ncu, committed under
    profiles/), or None when no capture has been summarised."""
    p = ROOT / "profiles" / "alpha_kernel_traffic.json"
    if not p.exists():
        return None
    d = json.loads(p.read_text())
    return float(d["dram_bytes"]) / float(d["alg_bytes"])


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = Path(os.environ.get("TMPDIR", "/tmp")) / f"specann_clocks_{os.getpid()}.csv"

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        for line in self.path.read_text().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            for name, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        try:
            self.path.unlink()
        except Exception:
            pass
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": float(max(smax)) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def make_graph(args, seed=42):
    from specann_b200 import graphs
    n = 1 << args.log2n
    rowptr, col, val = graphs.barabasi_albert_arrays(n, args.m, seed=seed, couplings="unit")
    return n, rowptr, col, val


def spmv_bytes(n, nnz, rp_bytes, t):
    """Algorithmic bytes of one fused SpMV: nnz (col + value) + (n+1) row pointers + x, s, y."""
    return nnz * (4 + t) + (n + 1) * rp_bytes + 3 * n * t


def pinned_csr(J, keep):
    """A CSR over copies of J's arrays in page-locked host memory (the e2e inputs: the copies inside
    the timed region are then DMA transfers, not pageable copies staged by the CPU). The pinned
    tensors are appended to `keep`. Returns (CSR, whether SciPy kept the pinned arrays uncopied)."""
    import scipy.sparse as sp
    import torch
    arrs = []
    for a in (J.data, J.indices, J.indptr):
        t_ = torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
        keep.append(t_)
        arrs.append(t_.numpy())
    P = sp.csr_matrix((arrs[0], arrs[1], arrs[2]), shape=J.shape)
    return P, all(np.shares_memory(x, y) for x, y in zip((P.data, P.indices, P.indptr), arrs))


def workload_name(args):
    """The workload string both arms print."""
    return (f"BA(n=2^{args.log2n}, m={args.m}) J=-A, {args.num_alphas} alphas sqrt schedule, diagonal predictor, "
            f"eigsh_tol 1e-6, batched local search")


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def blas_threads():
    """BLAS / OpenMP thread pools of this process (threadpoolctl), for the CPU baseline's record."""
    try:
        from threadpoolctl import threadpool_info
        return [{"api": d.get("user_api"), "lib": d.get("internal_api"), "threads": d.get("num_threads")}
                for d in threadpool_info()]
    except Exception as e:      # threadpoolctl missing: say so
        return [{"error": str(e)}]


def oracle_graph(args):
    """(n, rowptr int64, col int32, val float32) of the benchmark graph, written by the oracle's
    stand-alone executable (oracle/_bin/ba_graph, built from the same generator source), so that the
    CPU reference process loads none of the product's libraries."""
    import tempfile
    from oracle import build_tools
    exe = build_tools.BIN if build_tools.BIN.exists() else build_tools.build()
    n = 1 << args.log2n
    with tempfile.TemporaryDirectory() as tmp:
        path = Path(tmp) / "graph.bin"
        subprocess.run([str(exe), "ba", str(n), str(args.m), "42", "0", str(path)], check=True)
        raw = np.fromfile(path, dtype=np.uint8)
    n_, nnz = np.frombuffer(raw[:16], dtype=np.int64)
    o = 16
    rowptr = np.frombuffer(raw[o:o + 8 * (n_ + 1)], dtype=np.int64)
    o += 8 * (int(n_) + 1)
    col = np.frombuffer(raw[o:o + 4 * nnz], dtype=np.int32)
    o += 4 * int(nnz)
    val = np.frombuffer(raw[o:o + 4 * nnz], dtype=np.float32)
    return int(n_), rowptr, col, val


class CpuSweep:
    """The oracle's sweep of the benchmark workload (SciPy ARPACK eigsh + NumPy local search on
    `threads` host threads), advanced alpha by alpha in schedule order with the reference's warm-start
    chain (models/spectral_annealing.py:568-669): only alpha 0 starts cold. `timed_alpha(t)` solves
    alpha t - 1 untimed (warm-started from wherever the chain is) and then times alpha t, warm-started
    from its true predecessor, as in a full sweep."""

    def __init__(self, J, num_alphas, threads, seed=42):
        from oracle import specann_oracle as O
        self.O = O
        self.J = J
        self.pre = O.prelude(J, 32, threads=threads)
        self.alphas = O.alpha_schedule("sqrt", num_alphas)
        self.rng = np.random.default_rng(seed)
        self.threads = threads
        self.pos = -1
        self.y_last = self.y_prev = self.lam = self.a_prev = None
        self.spins = []

    def _advance(self, i):
        res = self.O.solve_alpha(self.pre, self.alphas[i], i, self.a_prev, self.y_last, self.y_prev, self.lam,
                                 rng=self.rng)
        self.y_prev, self.y_last = self.y_last, res.y
        self.lam, self.a_prev, self.pos = res.lambda1, self.alphas[i], i
        return res

    def timed_alpha(self, t):
        if self.pos < t - 1:
            self._advance(t - 1)
        t0 = time.perf_counter()
        res = self._advance(t)
        dt = time.perf_counter() - t0
        self.spins.append(self.O.round_spins(res.x))
        return dt

    def timed_ls_pass(self, k, seed):
        """Seconds per local-search pass over k candidates: two main-loop passes over k candidates (the
        rounded spins of the timed alphas, padded with seeded perturbations of them) divided by 3 (the
        initial field product costs about one pass), a slight underestimate of a pass."""
        base = self.spins[-1] if self.spins else np.ones(self.J.shape[0], dtype=np.int8)
        rng = np.random.default_rng(seed)
        S = [s for s in self.spins[-k:]]
        while len(S) < k:
            flip = rng.random(base.size) < 0.05
            S.append(np.where(flip, -base, base).astype(np.int8))
        t0 = time.perf_counter()
        self.O.local_search(self.J, np.stack(S), seed=seed, max_iterations=2, num_rounds=0, threads=self.threads)
        return (time.perf_counter() - t0) / 3.0


def spread_targets(count, num_alphas):
    """`count` alpha indices spread evenly over 1 .. num_alphas - 1 (alpha 0, the cold start, excluded)."""
    if count <= 1:
        return [num_alphas // 2]
    return [1 + int(round(s * (num_alphas - 2) / (count - 1))) for s in range(count)]


def cpu_solve_estimate(sweep, t_alpha, t_pass, k_ls, args):
    """One full solve from one timed alpha and one timed local-search pass: num_alphas x the alpha's
    time + (candidates x passes of a full solve) x the per-candidate pass time."""
    return t_alpha * args.num_alphas + t_pass / k_ls * args.ref_candidates * args.ref_ls_passes


def run_reference(args, rank, world):
    """The reference arm: the CPU reference pipeline (the oracle port; the reference's own path is
    CuPy-only) on the same workload, one alpha of the sweep per step, spread over the schedule. Each
    step times one alpha warm-started from its true predecessor plus one local-search pass, and is
    extrapolated to a full solve (cpu_solve_estimate); `value` is the mean over the timed steps. Under
    torchrun only rank 0 runs."""
    if rank != 0:
        return
    import scipy.sparse as sp
    n, rowptr, col, val = oracle_graph(args)
    J = sp.csr_matrix((val.astype(np.float64), col, rowptr), shape=(n, n))
    threads = host_threads()
    sweep = CpuSweep(J, args.num_alphas, threads)
    targets = spread_targets(args.warmup + args.steps, args.num_alphas)
    k_ls = 16
    est, t_alphas, t_passes = [], [], []
    for step, t in enumerate(targets):
        ta = sweep.timed_alpha(t)
        tp = sweep.timed_ls_pass(k_ls, seed=42 + step)
        if step >= args.warmup:
            est.append(cpu_solve_estimate(sweep, ta, tp, k_ls, args))
            t_alphas.append(ta)
            t_passes.append(tp)
    value = float(np.mean(est))
    timed = targets[args.warmup:]
    sample = (f"per step one alpha of the {args.num_alphas}-alpha sqrt sweep (indices {timed[0]}..{timed[-1]}, "
              f"spread evenly; each warm-started from its true predecessor, solved untimed just before) x "
              f"{args.num_alphas}, mean {np.mean(t_alphas):.3f} s/alpha; plus one local-search pass over {k_ls} "
              f"candidates ({np.mean(t_passes):.3f} s) scaled to {args.ref_candidates} candidates x "
              f"{args.ref_ls_passes} passes (the GPU solve's counts; its local search is bit-exact with this one); "
              f"SciPy ARPACK eigsh + NumPy, sparse products on {threads} threads")
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": value * 1000.0, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32" if args.precision == 32 else "f64",
            "data": "synthetic (seeded BA generator, J = -A)", "impl": "reference",
            "config": {"workload": workload_name(args), "n": n, "nnz": int(rowptr[-1])},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample,
                             "host_cpu_count": os.cpu_count(), "blas": blas_threads(),
                             "extrapolation": f"x{args.num_alphas} per alpha; local search x"
                                              f"{args.ref_candidates * args.ref_ls_passes / k_ls:g} per pass"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def cpu_baseline_sample(args, J, k_gpu, passes_gpu, count=4):
    """The ours arm's CPU baseline: the oracle sweep on a bounded sample (`count` alphas spread over the
    schedule, each warm-started from its true predecessor, plus one local-search pass each), extrapolated
    to one full solve with the GPU solve's candidate and pass counts."""
    threads = host_threads()
    sweep = CpuSweep(J, args.num_alphas, threads)
    k_ls = 16
    targets = spread_targets(count, args.num_alphas)
    ta, tp = [], []
    t_all = time.perf_counter()
    for i, t in enumerate(targets):
        ta.append(sweep.timed_alpha(t))
        tp.append(sweep.timed_ls_pass(k_ls, seed=42 + i))
    wall = time.perf_counter() - t_all
    value = float(np.mean(ta)) * args.num_alphas + float(np.mean(tp)) / k_ls * k_gpu * passes_gpu
    return {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{count} alphas of the {args.num_alphas}-alpha sqrt sweep (indices {targets}), each "
                      f"warm-started from its true predecessor (solved untimed), mean {np.mean(ta):.3f} s/alpha "
                      f"x{args.num_alphas}; one local-search pass over {k_ls} candidates per alpha "
                      f"({np.mean(tp):.3f} s) scaled to the GPU solve's {k_gpu} candidates x {passes_gpu} passes; "
                      f"SciPy ARPACK eigsh + NumPy, sparse products on {threads} threads ({wall:.0f} s of CPU work)",
            "host_cpu_count": os.cpu_count(), "blas": blas_threads()}


def full_solve_baselines(args):
    """Whole 128-alpha solves of the two small configurations on both sides: C1 (ER(1024, 20/1023),
    linear schedule) and C2 (BA(2^16, 20), sqrt schedule), local search on, seed 42. The CPU side is
    the oracle pipeline on all host threads; the GPU side is SpectralAnnealing.solve on the host CSR
    (its uploads inside the time)."""
    import torch
    from oracle import specann_oracle as O
    from specann_b200 import graphs
    from specann_b200.spectral_annealing import SpectralAnnealing
    threads = host_threads()
    cases = {"C1 ER(1024, p=20/1023) linear x128": (graphs.erdos_renyi(1024, 20 / 1023, seed=42), "linear"),
             "C2 BA(2^16, m=20) sqrt x128": (graphs.barabasi_albert(1 << 16, 20, seed=42), "sqrt")}
    out = {}
    for name, (J, sched) in cases.items():
        SpectralAnnealing("w.txt", "w", random_seed=42, schedule=sched, num_alphas=4, write_results=False).solve(J)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e_gpu, _, _ = SpectralAnnealing("f.txt", "f", random_seed=42, schedule=sched, write_results=False).solve(J)
        torch.cuda.synchronize()
        t_gpu = time.perf_counter() - t0
        t0 = time.perf_counter()
        res = O.solve(J, seed=42, schedule=sched, num_alphas=args.num_alphas, threads=threads)
        t_cpu = time.perf_counter() - t0
        out[name] = {"gpu_s": t_gpu, "cpu_s": t_cpu, "cpu_cores": threads, "gpu_best_energy": e_gpu,
                     "cpu_best_energy": res.best_energy}
    return out


def run_batch(args, rank, world, local):
    """The ragged batched workload: 64 instances (n log-uniform in [2^10, 2^17], half ER degree 20,
    half BA m 10/20, +-1 couplings) x 4 seeds x 128 alphas in one launch per GPU. Under torchrun the
    instances are sharded over the ranks (strong scaling: the total work is fixed); the time is the
    max over ranks."""
    import torch
    import torch.distributed as dist
    from specann_b200 import _lib, graphs, sharding
    from specann_b200.batch import BatchedSpectralAnnealing
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    dev = torch.device("cuda", local)
    lib = _lib.load()
    inst = graphs.ragged_batch(count=args.batch_count)
    Js = [J for _, J in inst]
    seeds = (42, 43, 44, 45)
    mine = sharding.shard_instances([(J.shape[0], J.nnz) for J in Js], world)[rank]
    mJs = [Js[i] for i in mine]
    b = BatchedSpectralAnnealing(seeds=seeds, num_alphas=args.num_alphas)
    b.load(mJs)
    tune = b.autotune(splits=(1.0, 2.0, 4.0), num_alphas=8)
    for _ in range(args.warmup):
        b.sweep()
    clocks = ClockSampler(local)
    launches0 = lib.sa_kernel_launches()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    times = [b.sweep() for _ in range(args.steps)]
    clk = clocks.stop()
    launches = lib.sa_kernel_launches() - launches0
    ms = float(np.mean(times))
    res = b.results()
    if world > 1:
        tt = torch.tensor([ms], device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms = float(tt.item())
    spmvs = sum(r2["eigsh_spmvs"] for r in res for r2 in r["rows"])
    alg = 0.0
    for r in res:
        J = mJs[r["instance"]]
        per = J.nnz * 8 + (J.shape[0] + 1) * 4 + 12 * J.shape[0]
        alg += per * sum(x["eigsh_spmvs"] for x in r["rows"])
    hbm, kind = peaks()
    # e2e: host CSRs (page-locked) -> upload + preludes -> batched launch -> best spins back, through
    # the public API
    pinned_keep = []
    pJs = [pinned_csr(J, pinned_keep) for J in mJs]
    h2d_pinned = all(ok for _, ok in pJs)
    pJs = [P for P, _ in pJs]
    t0 = time.perf_counter()
    e2 = BatchedSpectralAnnealing(seeds=seeds, num_alphas=args.num_alphas, split=b._built_split)
    out = e2.solve(pJs)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    e2.close()
    if world > 1:
        tt = torch.tensor([e2e_s], device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_s = float(tt.item())
    h2d = int(sum(J.indptr.size * 4 + J.nnz * 8 for J in mJs))
    d2h = int(sum(J.shape[0] for J in mJs) * len(seeds) // 8)
    line = {"metric": "s per ragged batch (64 instances x 4 seeds x 128 alphas, one launch per GPU)",
            "value": ms / 1000.0, "unit": "s/batch", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms, "higher_is_better": False, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded ER/BA generators, +-1 couplings)",
            "config": {"workload": "ragged batch: 64 instances, n log-uniform 2^10..2^17, half ER deg 20, half BA "
                                   "m 10/20, 4 seeds x 128 alphas sqrt, diagonal predictor, batched LS",
                       "instances_on_rank0": len(mJs), "problems": len(mJs) * len(seeds),
                       "total_nnz": int(sum(J.nnz for J in Js)), "teams": int(len(b.team_b0)),
                       "largest_team": int(b.team_nb.max()), "grid": b.grid(), "autotune_ms": tune,
                       "split": b._built_split, "graph": True,
                       "l2": "working set of the batch (CSR + bases) larger than L2"},
            "e2e": {"value": e2e_s, "unit": "s/batch", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "h2d_source": "pinned host memory" if h2d_pinned else "pageable host memory"},
            "roofline": {"bound": "hbm", "achieved": alg / (ms / 1e3) / 1e9, "peak": hbm, "unit": "GB/s",
                         "frac": alg / (ms / 1e3) / 1e9 / hbm, "traffic": None, "peak_source": kind,
                         "kernel": "batch_kernel (SpMV bytes only: a lower bound of its traffic)",
                         "spmvs": spmvs},
            "problems_ok": int(sum(1 for r in res if r["status"] == 0)),
            "cta_utilization": float(sum(r["device_ms"] * r["team"][1] for r in res) / (ms * b.grid())),
            "problem_device_ms": {"max": float(max(r["device_ms"] for r in res)),
                                  "sum": float(sum(r["device_ms"] for r in res))},
            "clocks": clk, "gpu_launches": int(launches)}
    if rank == 0:
        print(json.dumps(line))
    b.close()
    if world > 1:
        dist.destroy_process_group()


def run_precision(args):
    """Precision form on BA(2^16, m 20), J = -A: FP32 SpMV/Lanczos with FP64 Ritz and residual
    against the all-FP64 path, per alpha (eigenvalue error, residual, raw energy) and best energy."""
    from specann_b200 import graphs
    from specann_b200.spectral_annealing import SpectralAnnealing
    J = graphs.barabasi_albert(1 << 16, 20, seed=42)
    for prec in (32, 64):    # load the library and kernels once (not timed)
        SpectralAnnealing("w.txt", "w", random_seed=1, precision=prec, num_alphas=4, write_results=False).solve(J)
    runs = {}
    for prec in (32, 64):
        s = SpectralAnnealing("c2.txt", "c2", random_seed=42, precision=prec, write_results=False, profile=True)
        t0 = time.perf_counter()
        e, spins, _ = s.solve(J)
        dt = time.perf_counter() - t0
        runs[prec] = (s, e, dt)
    r32, r64 = runs[32][0].alpha_results, runs[64][0].alpha_results
    lam_err = np.array([abs(a["lambda1"] - b["lambda1"]) for a, b in zip(r32, r64)])
    res32 = np.array([a["eigsh_residual"] for a in r32])
    res64 = np.array([b["eigsh_residual"] for b in r64])
    raw_gap = np.array([abs(a["raw_energy"] - b["raw_energy"]) / abs(b["raw_energy"]) for a, b in zip(r32, r64)])
    same = sum(1 for a, b in zip(r32, r64) if a["raw_energy"] == b["raw_energy"])
    out = {"workload": "precision: BA(2^16, m=20) J=-A, 128 alphas sqrt, seed 42",
           "fp32_s": runs[32][2], "fp64_s": runs[64][2], "best_fp32": runs[32][1], "best_fp64": runs[64][1],
           "best_gap_rel": abs(runs[32][1] - runs[64][1]) / abs(runs[64][1]),
           "lambda_abs_err": {"max": float(lam_err.max()), "median": float(np.median(lam_err))},
           "residual_fp32": {"max": float(np.nanmax(res32)), "median": float(np.nanmedian(res32))},
           "residual_fp64": {"max": float(np.nanmax(res64)), "median": float(np.nanmedian(res64))},
           "raw_energy_gap_rel": {"max": float(raw_gap.max()), "median": float(np.median(raw_gap))},
           "alphas_same_raw_energy": same, "spmvs_fp32": runs[32][0].engine.stats["spmvs"],
           "spmvs_fp64": runs[64][0].engine.stats["spmvs"],
           "per_alpha": [{"alpha": a["alpha"], "lambda_fp32": a["lambda1"], "lambda_fp64": b["lambda1"],
                          "res_fp32": a["eigsh_residual"], "res_fp64": b["eigsh_residual"],
                          "raw_fp32": a["raw_energy"], "raw_fp64": b["raw_energy"]} for a, b in zip(r32, r64)]}
    print(json.dumps(out))


def run_grad(args):
    """Differentiation form on BA(2^18, m 20), +-1 couplings, beta 8: adjoint gradient time and its
    central-FD check (h 1e-4, FP64), and Lanczos work per alpha of the three predictors."""
    import torch
    from specann_b200 import _lib, graphs
    from specann_b200.differentiation import EigenProblem
    from specann_b200.spectral_annealing import SpectralAnnealing
    J = graphs.barabasi_albert(1 << 18, 20, seed=42, couplings="pm1")
    out = {"workload": "grad: BA(2^18, m=20) +-1 couplings, beta 8"}
    for prec, tol, atol in ((32, 1e-6, 1e-4), (64, 1e-10, 1e-8)):
        prob = EigenProblem(J, precision=prec)
        prob.energy_and_gradient(0.5, beta=8.0, tol=tol, adj_tol=atol)        # warm-up
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        lam, y = prob.eigenpair(0.5, tol=tol)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        grad = torch.empty(prob.n, dtype=torch.float64, device="cuda")
        res = prob.engine.adjoint(_lib.SA_ADJ_GRADIENT, alpha=0.5, lambda1=lam, y=y, beta=8.0, tol=atol, maxiter=4000, grad=grad)
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        d = {"eig_s": t1 - t0, "adjoint_s": t2 - t1, "minres_iterations": res.iterations,
             "minres_residual": res.residual, "loss": res.loss, "dL_dalpha": res.dloss_dalpha}
        if prec == 64:
            h = 1e-4
            Lp = prob.energy_and_gradient(0.5 + h, beta=8.0, tol=tol, adj_tol=1e-2)[0]
            Lm = prob.energy_and_gradient(0.5 - h, beta=8.0, tol=tol, adj_tol=1e-2)[0]
            d["fd"] = (Lp - Lm) / (2 * h)
            d["fd_rel_err"] = abs(d["fd"] - res.dloss_dalpha) / abs(d["fd"])
        out[f"fp{prec}"] = d
        prob.close()
    pred = {}
    for mode in ("diagonal", "secant", "tangent"):
        s = SpectralAnnealing("c4.txt", "c4", random_seed=42, pred_mode=mode, write_results=False,
                              use_local_search=False)
        t0 = time.perf_counter()
        e, _, _ = s.solve(J)
        dt = time.perf_counter() - t0
        rows = s.alpha_results
        it = np.array([r["eigsh_iterations"] for r in rows])
        pred[mode] = {"s": dt, "best_raw_energy": e, "lanczos_iters_mean": float(it.mean()),
                      "lanczos_iters_median": float(np.median(it)), "lanczos_spmvs": int(sum(r["eigsh_spmvs"] for r in rows)),
                      "tangent_spmvs": int(sum(r.get("tangent_spmvs", 0) for r in rows)),
                      "pred_accepted": int(sum(1 for r in rows if r["pred_accepted"]))}
    out["predictors"] = pred
    print(json.dumps(out))


def scale_solves(args, dev, n, rowptr, col, val, d_rowptr=None, d_col=None, d_val=None):
    """One timed FP32 (FP64 Ritz) solve and one timed all-FP64 solve of the same graph, CSR resident
    (int64 row pointers, int32 columns), and their best-energy gap: the large-scale half of the metric.
    Returns the block as a dict; frees its device arrays."""
    import torch
    from specann_b200.spectral_annealing import SpectralAnnealing
    nnz = int(rowptr[-1])
    if d_rowptr is None:
        d_rowptr = torch.from_numpy(np.ascontiguousarray(rowptr, dtype=np.int64)).to(dev)
        d_col = torch.from_numpy(col).to(dev)
        d_val = torch.from_numpy(val).to(dev)
    out = {"n": n, "nnz": nnz, "rowptr": str(d_rowptr.dtype).replace("torch.", ""),
           "workload": f"BA(n={n}, m={args.m}) J=-A, {args.num_alphas} alphas sqrt schedule, diagonal predictor, "
                       f"eigsh_tol 1e-6, eigsh_maxiter {args.scale_maxiter}, batched local search; CSR resident"}
    from specann_b200 import graphs as _g
    Jw = _g.barabasi_albert(4096, 8, seed=1)       # load the kernels once (not timed)
    SpectralAnnealing("w.txt", "w", random_seed=1, num_alphas=4, write_results=False).solve(Jw)
    for prec in [int(x) for x in args.scale_precisions.split(",")]:
        if prec == 64:
            del d_val
            torch.cuda.empty_cache()
            d_val = torch.from_numpy(val.astype(np.float64)).to(dev)
        s = SpectralAnnealing("scale.txt", "scale", random_seed=42, num_alphas=args.num_alphas, precision=prec,
                              eigsh_maxiter=args.scale_maxiter, write_results=False, profile=True)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e, spins, _ = s.solve_device(d_rowptr, d_col, d_val)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        st = s.engine.stats
        iters = [r["eigsh_iterations"] for r in s.alpha_results]
        res = [r["eigsh_residual"] for r in s.alpha_results]
        out[f"fp{prec}"] = {"seconds": dt, "best_energy": e, "spmvs": st["spmvs"], "layout": s.operator_layout,
                            "alpha_kernel_s": st["alpha_ms"] / 1e3, "ls_kernel_s": st["ls_ms"] / 1e3,
                            "alpha_GBps": st["alpha_bytes"] / (st["alpha_ms"] / 1e3) / 1e9,
                            "phase_s": [round(x / 1e3, 3) for x in st.get("phase_ms", [0] * 6)],
                            "iters_mean": float(np.mean(iters)), "iters_max": int(np.max(iters)),
                            "max_residual": float(np.nanmax(res)),
                            "alphas_above_1e-5": int(sum(1 for x in res if x > 1e-5)),
                            # alphas that stopped at maxiter unconverged (the reference marks
                            # them "energy bound not certified" and keeps them)
                            "uncertified": [{"alpha_index": r["alpha_index"], "alpha": r["alpha"],
                                             "iterations": r["eigsh_iterations"],
                                             "residual": r["eigsh_residual"],
                                             "cold_start": r["alpha_index"] == 0}
                                            for r in s.alpha_results if not r["eigsh_converged"]],
                            "alphas_skipped": int(s._alphas_skipped),
                            "candidates": int(s._num_candidates or 0),
                            "peak_mem_gb": torch.cuda.max_memory_allocated() / 1e9}
        del s
        torch.cuda.empty_cache()
    if "fp32" in out and "fp64" in out:
        e32, e64 = out["fp32"]["best_energy"], out["fp64"]["best_energy"]
        out["energy_gap_rel"] = abs(e32 - e64) / abs(e64)
        out["fp64_over_fp32"] = out["fp64"]["seconds"] / out["fp32"]["seconds"]
    del d_rowptr, d_col, d_val
    torch.cuda.empty_cache()
    return out


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.workload == "batch":
        run_batch(args, rank, world, local)
        return
    if args.workload == "precision":
        run_precision(args)
        return
    if args.workload == "grad":
        run_grad(args)
        return
    import torch
    import torch.distributed as dist
    from specann_b200 import _lib
    from specann_b200.spectral_annealing import SpectralAnnealing

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    dev = torch.device("cuda", local)
    lib = _lib.load()
    n, rowptr, col, val = make_graph(args)
    nnz = int(rowptr[-1])
    # 64-bit row pointers for the scale run (the C5 form: int32 columns, int64 row pointers) or when nnz
    # needs them; else int32
    rp_np = rowptr if (args.scale_run or nnz >= 2**31) else rowptr.astype(np.int32)
    import scipy.sparse as sp
    # the e2e input: a SciPy CSR whose arrays live in page-locked host memory
    pinned_keep = []
    J_host, h2d_pinned = pinned_csr(
        sp.csr_matrix((val.astype(np.float64) if args.precision == 64 else val, col, rp_np), shape=(n, n)),
        pinned_keep)
    d_rowptr = torch.from_numpy(rp_np).to(dev)
    d_col = torch.from_numpy(col).to(dev)
    d_val = torch.from_numpy(val if args.precision == 32 else val.astype(np.float64)).to(dev)
    t = 4 if args.precision == 32 else 8
    seed = 42 + rank

    def solver(profile=False):
        return SpectralAnnealing("bench.txt", "bench", random_seed=seed, num_alphas=args.num_alphas,
                                 precision=args.precision, write_results=False, profile=profile)

    def barrier():
        if world > 1:
            dist.barrier()

    if args.scale_run:
        out = scale_solves(args, dev, n, rowptr, col, val, d_rowptr, d_col, d_val)
        print(json.dumps(out))
        return

    if args.spmv_only:
        from specann_b200.engine import Engine
        eng = Engine(n, nnz, precision=args.precision, ncv_max=33, max_candidates=1)
        eng.bind(d_rowptr, d_col, d_val)
        layout = args.spmv_layout
        if layout == "auto":
            layout = "panel" if eng.panels_pay() else ("split" if eng.splits_pay() else "worklist")
        if layout == "panel":
            eng.build_panels()
        elif layout == "split":
            eng.build_splits()
        x = torch.randn(n, device=dev, dtype=torch.float32 if args.precision == 32 else torch.float64)
        y = torch.empty_like(x)
        for _ in range(args.warmup):
            eng.spmv(0.5, 1.001, x, y)
        torch.cuda.synchronize()
        s0 = torch.cuda.Event(enable_timing=True)
        s1 = torch.cuda.Event(enable_timing=True)
        s0.record()
        for _ in range(args.spmv_reps):
            eng.spmv(0.5, 1.001, x, y)
        s1.record()
        torch.cuda.synchronize()
        ms_ = s0.elapsed_time(s1) / args.spmv_reps
        sb_ = spmv_bytes(n, nnz, rp_np.itemsize, t)
        hbm_, kind_ = peaks()
        print(json.dumps({"spmv_only": True, "layout": layout, "n": n, "nnz": nnz, "ms": ms_, "bytes": sb_,
                          "GBps": sb_ / ms_ / 1e6, "frac": sb_ / ms_ / 1e6 / hbm_, "peak_source": kind_}))
        return

    # warm-up (untimed), then K timed steps with the CSR resident in HBM
    for _ in range(args.warmup):
        solver().solve_device(d_rowptr, d_col, d_val)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    stream = torch.cuda.current_stream()
    launches0 = lib.sa_kernel_launches()
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    energies = []
    for _ in range(args.steps):
        e, _, _ = solver().solve_device(d_rowptr, d_col, d_val)
        energies.append(e)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    launches = lib.sa_kernel_launches() - launches0
    ms = e0.elapsed_time(e1) / args.steps
    if world > 1:
        tt = torch.tensor([ms], device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms = float(tt.item())
    value = ms / 1000.0 / world

    # one profiled solve: per-kernel event times and algorithmic bytes of the alpha kernels
    s = solver(profile=True)
    s.solve_device(d_rowptr, d_col, d_val)
    st = s.engine.stats
    iters = np.array([r["eigsh_iterations"] for r in s.alpha_results], dtype=np.float64)
    if os.environ.get("SPECANN_BENCH_DUMP"):
        with open(os.environ["SPECANN_BENCH_DUMP"], "w") as f:
            for r in s.alpha_results:
                f.write(json.dumps({k: r[k] for k in ("alpha", "eigsh_iterations", "eigsh_restarts", "eigsh_residual",
                                                      "lambda1", "pred_accepted", "pred_residual", "candidate",
                                                      "eigsh_spmvs", "alg_bytes")}) + "\n")
    lanczos = {"mean": float(iters.mean()), "median": float(np.median(iters)), "max": float(iters.max()),
               "alpha0": float(iters[0]), "restarts": int(sum(r["eigsh_restarts"] for r in s.alpha_results)),
               "pred_accepted": int(sum(1 for r in s.alpha_results if r["pred_accepted"])),
               "max_residual": float(np.nanmax([r["eigsh_residual"] for r in s.alpha_results])),
               "candidates": int(s._num_candidates or 0), "ls_passes": int(getattr(s, "_ls_passes", 0))}
    hbm, peak_kind = peaks()
    alpha_gbs = st["alpha_bytes"] / (st["alpha_ms"] / 1000.0) / 1e9 if st["alpha_ms"] > 0 else None

    # standalone fused SpMV (the north-star SpMV bandwidth figure): K launches on resident data
    from specann_b200.engine import Engine
    eng = Engine(n, nnz, precision=args.precision, ncv_max=33, max_candidates=1)
    eng.bind(d_rowptr, d_col, d_val)
    layout = getattr(s, "operator_layout", "worklist")
    # algorithmic bytes of one application (the CSR formula: nnz (col + value) + row pointers + x, s,
    # y); the layout's own stream (packed panel words, split partial sums) is reported beside it
    sb = spmv_bytes(n, nnz, rp_np.itemsize, t)
    stream_b = sb
    if layout == "panel":
        eng.build_panels()
        stream_b = eng.panel_info()["matrix_bytes"] + 3 * n * t
    elif layout == "split":
        eng.build_splits()
        stream_b = eng.split_bytes() + 3 * n * t
    x = torch.randn(n, device=dev, dtype=torch.float32 if args.precision == 32 else torch.float64)
    y = torch.empty_like(x)
    for _ in range(3):
        eng.spmv(0.5, 1.001, x, y)
    torch.cuda.synchronize()
    s0 = torch.cuda.Event(enable_timing=True)
    s1 = torch.cuda.Event(enable_timing=True)
    s0.record(stream)
    for _ in range(args.spmv_reps):
        eng.spmv(0.5, 1.001, x, y)
    s1.record(stream)
    torch.cuda.synchronize()
    spmv_ms = s0.elapsed_time(s1) / args.spmv_reps   # includes the O(n) scale kernel of each call
    spmv_gbs = sb / (spmv_ms / 1000.0) / 1e9

    # e2e: the public API with a host SciPy CSR (H2D of the matrix and D2H of the spins inside)
    e2e_steps = args.e2e_steps or max(1, min(args.steps, 3))
    torch.cuda.synchronize()
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        solver().solve(J_host)
    torch.cuda.synchronize()
    e2e_s = (time.perf_counter() - t0) / e2e_steps
    if world > 1:
        tt = torch.tensor([e2e_s], device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_s = float(tt.item())
    h2d = int(rp_np.nbytes + col.nbytes + nnz * (4 if args.precision == 32 else 8))
    d2h = int(n * t)

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32" if args.precision == 32 else "f64",
        "data": "synthetic (seeded BA generator, J = -A)",
        "config": {"workload": workload_name(args),
                   "n": n, "nnz": nnz, "precision": args.precision, "replicas": world,
                   "l2": "inputs larger than L2 (CSR %.0f MB > 126 MB)" % ((rp_np.nbytes + col.nbytes + nnz * t) / 1e6),
                   "best_energy": float(energies[-1]) if energies else None},
        "e2e": {"value": e2e_s / world, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "h2d_source": "pinned host memory" if h2d_pinned else "pageable host memory"},
        "roofline": {"bound": "hbm", "achieved": alpha_gbs, "peak": hbm, "unit": "GB/s",
                     "frac": (alpha_gbs / hbm) if alpha_gbs else None,
                     "traffic": (traffic_ratio() * st["alpha_bytes"] / max(1, st["alpha_launches"]))
                     if traffic_ratio() else None,
                     "traffic_note": "bytes per alpha_kernel launch: the DRAM/algorithmic ratio of one ncu "
                                     "capture (profiles/alpha_kernel_traffic.json) times this run's mean "
                                     "algorithmic bytes per launch",
                     "alg_bytes_per_launch": st["alpha_bytes"] / max(1, st["alpha_launches"]),
                     "kernel": "alpha_kernel (persistent: fused SpMV + Lanczos + rounding)",
                     "peak_source": peak_kind,
                     "alpha_kernel_ms_per_solve": st["alpha_ms"], "alpha_launches_per_solve": st["alpha_launches"],
                     "spmvs_per_solve": st["spmvs"], "ls_kernel_ms_per_solve": st["ls_ms"],
                     "ls_phase_ms": dict(zip(("setup", "decide", "scatter", "final"),
                                            [round(x, 3) for x in st.get("ls_phase_ms", [0.0] * 4)])),
                     "alpha_phase_ms": dict(zip(("setup", "spmv", "dots", "update_ritz", "restart", "final"),
                                               [round(x, 3) for x in st.get("phase_ms", [0.0] * 6)])),
                     "lanczos_iterations": lanczos},
        "spmv": {"achieved": spmv_gbs, "peak": hbm, "unit": "GB/s", "frac": spmv_gbs / hbm,
                 "ms": spmv_ms, "bytes": sb, "layout": layout, "layout_stream_bytes": stream_b},
        "clocks": clk,
        "gpu_launches": int(launches),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_sample(args, J_host, int(s._num_candidates or 1),
                                                   int(getattr(s, "_ls_passes", 1)))
        line["cpu_baseline"]["full_solves"] = full_solve_baselines(args)
    if rank == 0 and world == 1 and args.scale_log2n > 0:
        # the large-scale half of the metric: BA(2^25) FP32 vs plain FP64 on this GPU
        del eng, x, y
        torch.cuda.empty_cache()
        import argparse as _ap
        sargs = _ap.Namespace(**vars(args))
        sargs.log2n = args.scale_log2n
        n2, rp2, col2, val2 = make_graph(sargs)
        line["scale"] = scale_solves(sargs, dev, n2, rp2, col2, val2)
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
