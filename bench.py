"""Benchmark: plain-FP64 two-site H_eff matvec at chi = 2048 (U(1), J1-J2-sized MPO).

One step = one application of the two-site effective Hamiltonian
(psi·L, ·W1, ·W2, ·R: four contract! calls, ITensorMPS's order; the
association psi·L·(W1·W2)·R is timed beside it) on synthetic, seeded inputs with
the shapes of the chi = 2048 J1-J2 6x6-cylinder workload: 11 U(1) sectors with
a Gaussian dimension profile summing to 2048 and an MPO link of 38 channels
graded by charge {-2: 12, 0: 14, +2: 12}.  The headline runs the ragged block
format (every block at its sector extents); the reference's uniform format
(every sector zero-padded to 411) is timed beside it on the same entries.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Beside the headline the line carries the reference's zero-padded layout
(cropped inside contract! and not), the permute stage, CUDA-graph replay, one
Lanczos solve, the cuBLAS block-list baseline, the 3xTF32 tensor-core form,
the N = 16 centre-bond problem, the serving loop (DMRG solves at three arrival
rates, solves/s with p50/p99), the PXP chain (N = 64, chi = 256, MPO in COO
and aliased storage) and the J1-J2 6x6 cylinder DMRG to chi = 2048, and the
CPU baseline: the C++ restatement of the reference path (oracle/cpu_ref).

Prints one JSON line (rank 0).  `value` is whole-job matvecs/s with inputs
resident in HBM; `e2e` is the same through the public API with psi uploaded
from pinned host memory and H·psi read back every step.  Multi-GPU runs are
independent replicas (the matvec does not shard): no data-path collective.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "H_eff matvec/s (plain FP64, chi=2048)"
UNIT = "matvec/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--chi", type=int, default=2048)
    ap.add_argument("--seed", type=int, default=2026)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-budget-s", type=float, default=60.0)
    ap.add_argument("--leg", default="all", choices=["all", "mixed", "dmrg", "cpu", "pxp", "j1j2"],
                    help="mixed: only the 3xTF32 tensor-core chain (psi*L*(W1*W2)*R, FP32 intermediates), "
                         "a short case for kernel profiling; dmrg: the full two-site DMRG of the Heisenberg "
                         "chain (N=100, chi 64->512, 5 sweeps) in FP64 and in 3xTF32; cpu: the oracle port "
                         "of the reference's algorithm on the host cores at 1 thread and at all threads, for the "
                         "chi=2048 matvec and the N=16 chi=64 centre-bond matvec; each prints its own line, not "
                         "the headline; pxp: the PXP chain (N=64, chi=256, MPO in COO) H_eff matvec in FP64 and "
                         "3xTF32 and the MPO x MPS apply, with the oracle port on the host cores; j1j2: two-site DMRG "
                         "of the J1-J2 model on the 6x6 cylinder (N=36, maxdim to --j1j2-maxdim) in FP64 and "
                         "3xTF32")
    ap.add_argument("--dmrg-n", type=int, default=100)
    ap.add_argument("--j1j2-maxdim", type=int, default=2048)
    ap.add_argument("--j1j2-split", default="gram", choices=["svd", "gram"],
                    help="factorisation of the two-site split (qn.split_two_site_device method)")
    ap.add_argument("--j1j2-budget-s", type=float, default=150.0,
                    help="no new FP64 sweep starts after this many seconds (the schedule is cut there)")
    return ap.parse_args()


def workload(chi: int):
    from sparsebackends_b200 import qn
    charges = list(range(-10, 11, 2))
    left = qn.gaussian_sectors(chi, charges, width=2.0)
    mpo = qn.mpo_link({-2: 12, 0: 14, 2: 12})
    return qn.HeffLayout(left, left, mpo)


def host_tensors(layout, seed: int, with_ragged: bool = False):
    """Seeded operands.  Uniform (reference layout, zero-padded sectors) always;
    with ``with_ragged`` also the same entries stored unpadded per block."""
    from sparsebackends_b200 import qn
    rng = np.random.Generator(np.random.PCG64(seed))
    out, rag = {}, {}
    for name, scale in (("psi", 1.0), ("L", 0.05), ("W1", 0.3), ("W2", 0.3), ("R", 0.05)):
        keys, data, exts = qn.random_block_tensor(layout, name, rng, scale, ragged=True)
        if name == "psi":
            data /= np.linalg.norm(data)
        out[name] = (keys, qn.pad_ragged(layout, name, keys, data, exts))
        rag[name] = (keys, data, exts)
    return (out, rag) if with_ragged else out


# ── clocks during the timed region ───────────────────────────────────────

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "100",
                 "-i", str(self.gpu)], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
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
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ── FP64 tensor-core peak (not in MEASURED_PEAKS.json): measured live ────

def measured_hbm_gbs():
    """HBM copy bandwidth measured on this pool (MEASURED_PEAKS.json), else the fallback."""
    try:
        with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"])
    except (OSError, KeyError, ValueError):
        return 6650.0


# DRAM bytes (read + write) per launch from one ncu capture of this bench at the
# given chi (--metrics dram__bytes_read.sum,dram__bytes_write.sum), averaged
# over the captured launches of each kernel.  A constant of that capture (its
# date below), not a measurement of this run: it goes stale when the kernel
# changes.
TRAFFIC = {
    (2048, "k_gemm_f64"): (1121.8e6, "ncu capture of 2026-12-03, mean of the psi*L and R*T3 launches"),
    (2048, "k_gemm_thin"): (1315.3e6, "ncu capture of 2026-12-03, mean of the T1*W1 and T2*W2 launches"),
}


def traffic_per_launch(chi: int, kernel: str):
    t = TRAFFIC.get((chi, kernel))
    return None if t is None else {"bytes": t[0], "source": t[1], "kind": "constant from a dated capture"}


def cublas_block_lists(layout, steps: int = 10):
    """cuBLAS DGEMM (torch.matmul / addmm) on the block lists of the two
    tensor-bound H_eff steps, psi*L and R*T3: per output block one GEMM per
    matched pair, accumulated in pair order, on random operands of the same
    shapes (unpadded sector extents).  Returns ms per step for both steps
    together, eager and replayed from a CUDA graph."""
    import torch
    from sparsebackends_b200 import qn
    lab = layout.labels

    def ext(kv, x):
        q = qn.GRADE[x]
        return qn._link_of(layout, q).dims[kv[q] - 1]

    gen = torch.Generator(device="cuda").manual_seed(7)
    work, flops = [], 0
    for st in qn.chain_structure(layout):
        if st["C"] not in ("T1", "T4"):
            continue
        lc = lab[st["C"]]
        pc = len(lc) - layout.n2[st["C"]]
        cbs = {}
        for kv in st["pairs"]:
            m = int(np.prod([ext(kv, x) for x in st["keepA"]] or [1]))
            n = int(np.prod([ext(kv, x) for x in st["keepB"]] or [1]))
            k = int(np.prod([ext(kv, x) for x in st["red"]] or [1]))
            cbs.setdefault(tuple(kv[x] for x in lc[:pc]), []).append((m, n, k))
        for prs in cbs.values():
            m, n = prs[0][0], prs[0][1]
            ops = [(torch.randn((m, k), dtype=torch.float64, device="cuda", generator=gen),
                    torch.randn((k, n), dtype=torch.float64, device="cuda", generator=gen)) for _, _, k in prs]
            work.append((torch.empty((m, n), dtype=torch.float64, device="cuda"), ops))
            flops += sum(2 * m * n * k for _, _, k in prs)

    def run():
        for c, ops in work:
            torch.matmul(ops[0][0], ops[0][1], out=c)
            for x, y in ops[1:]:
                c.addmm_(x, y)

    def timed_ms(fn):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        for _ in range(steps):
            fn()
        e.record()
        e.synchronize()
        return s.elapsed_time(e) / steps

    for _ in range(3):
        run()
    torch.cuda.synchronize()
    eager = timed_ms(run)
    graph = torch.cuda.CUDAGraph()
    side = torch.cuda.Stream()
    with torch.cuda.stream(side):
        run()
        torch.cuda.synchronize()
        with torch.cuda.graph(graph):
            run()
    torch.cuda.synchronize()
    replay = timed_ms(graph.replay)
    del graph, work
    torch.cuda.empty_cache()
    return {"what": "cuBLAS DGEMM (torch.matmul / addmm) per output block and matched pair, on the psi*L and R*T3 "
                    "block lists of this workload (unpadded extents, random operands of the same shapes)",
            "gflop_per_step": flops / 1e9, "ms_per_step": eager, "tflops": flops / eager / 1e9,
            "graph_ms_per_step": replay, "graph_tflops": flops / replay / 1e9}


def permute_stage(ctx, L, hbm_peak, reps: int = 5):
    """The permute stage (permutedims, storage.jl:188-264) on the zero-padded
    environment L of this workload (tail (mlp, mwl, ml), at chi = 2048 (411,
    14, 411) in 31 blocks, 0.62 GB): one tail permutation per transpose
    kernel.  Bytes are the algorithmic 16 per element (read once, written
    once); at chi = 2048 every permute reads and writes far more than L2, so
    no flush is needed."""
    import sparsebackends_b200 as sb
    cases = [("contiguous runs (k_permute_runs)", (1, 2, 3, 4, 6, 5)),
             ("narrow transpose, 14-wide rows (k_permute_narrow)", (1, 2, 3, 5, 4, 6)),
             ("tiled transpose, rows of one axis (k_permute_tiled)", (1, 2, 3, 6, 4, 5)),
             ("tiled transpose, rows of two axes (k_permute_tiled)", (1, 2, 3, 6, 5, 4))]
    out = []
    for name, perm in cases:
        sb.permutedims(L, perm)
        ctx.synchronize()
        ctx.set_profiling(True)
        for _ in range(reps):
            sb.permutedims(L, perm)
        p = ctx.profile("permute")
        ctx.set_profiling(False)
        gbs = p["bytes"] / (p["ms"] * 1e-3) / 1e9 if p["ms"] > 0 else 0.0
        out.append({"case": name, "perm": list(perm), "ms": p["ms"] / reps, "gb_per_s": gbs,
                    "frac": gbs / hbm_peak if hbm_peak else None})
    i = L._info()
    gb = i["nkeys"] * i["blksize"] * 8 / 1e9
    tail = i["dims"][len(i["dims"]) - i["n2"]:]
    return {"tensor": f"uniform L, tail {tail}, {i['nkeys']} blocks, {gb:.2f} GB",
            "peak_gb_per_s": hbm_peak,
            "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)", "cases": out}


def serving_leg(seed: int, nreq: int = 24):
    """The serving loop (``sparsebackends_b200.serving``): a seeded stream of
    XXZ ground-state solves (Delta ~ U[0.5, 1.5], N ~ U{8..24}, chi_max ~
    log-uniform [8, 64], two-site DMRG from the Neel state, 4 sweeps, cutoff
    1e-10, krylovdim 3, maxiter 1; reduced from N <= 128, chi_max <= 1024 so that
    the leg takes under a minute).  The baseline is the plain FP64 form served
    one request at a time; the served forms keep 4 requests in flight (own
    contexts and streams, admission by memory footprint), FP64 and 3xTF32.
    Arrival rates: 0.5, 1 and 2 times the baseline's capacity."""
    from sparsebackends_b200 import serving
    reqs = serving.random_requests(nreq, seed)
    warm = serving.Server(slots=1)
    warm.run(serving.random_requests(2, seed + 1, n_range=(8, 8), chi_range=(8, 8)))
    first = serving.Server(slots=1).run(reqs)  # all arrive at t = 0: the one-at-a-time capacity
    cap = serving.summary(first)
    out = {"stream": f"{nreq} XXZ solves, Delta~U[0.5,1.5], N~U{{8..24}}, chi_max~logU[8,64], 4 sweeps, cutoff "
                     "1e-10, krylovdim 3, maxiter 1 (reduced from N<=128, chi_max<=1024)",
           "baseline_capacity_solves_per_s": cap["solves_per_s"], "rates": []}
    base = {r.rid: r.energy for r in first}
    for f in (0.5, 1.0, 2.0):
        rate = f * cap["solves_per_s"]
        stream = serving.poisson_arrivals(reqs, rate, seed + 7)
        row = {"arrival_rate_per_s": rate, "fraction_of_baseline_capacity": f}
        for name, server in (("fp64_one_at_a_time", serving.Server(slots=1)),
                             ("fp64_4_in_flight", serving.Server(slots=4)),
                             ("tf32x3_4_in_flight", serving.Server(slots=4, precision="tf32x3"))):
            res = server.run(stream)
            row[name] = serving.summary(res)
            row[name]["max_rel_energy_diff_vs_fp64"] = max(abs(r.energy - base[r.rid]) / abs(base[r.rid])
                                                           for r in res)
        out["rates"].append(row)
    return out


def fp64_peak_tflops():
    import torch
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = math.inf
    for _ in range(10):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        e.synchronize()
        best = min(best, s.elapsed_time(e))
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


def tf32_peak_tflops():
    """Dense TF32 tensor-core rate: torch.matmul float32 with TF32 allowed, 8192^3, best of 10."""
    import torch
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = True
    try:
        n = 8192
        a = torch.randn(n, n, dtype=torch.float32, device="cuda")
        b = torch.randn(n, n, dtype=torch.float32, device="cuda")
        for _ in range(2):
            torch.matmul(a, b)
        torch.cuda.synchronize()
        best = math.inf
        for _ in range(10):
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            torch.matmul(a, b)
            e.record()
            e.synchronize()
            best = min(best, s.elapsed_time(e))
        del a, b
        torch.cuda.empty_cache()
        return 2.0 * n ** 3 / (best * 1e-3) / 1e12
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev


def mixed_dmrg_energy(local: int):
    """Two-site DMRG of the N = 12 Heisenberg chain in FP64 and with the
    tensor-core (3xTF32) H_eff applies plus the FP64 Rayleigh-quotient
    correction, same schedule; energies against each other and exact
    diagonalisation of the 2Sz = 0 sector."""
    import sparsebackends_b200 as sb
    from sparsebackends_b200 import dmrg
    n, sched = 12, [8, 16, 32, 64, 64]
    out = {"model": f"Heisenberg chain N={n}, OBC, U(1) 2Sz=0, chi schedule {sched}, cutoff 1e-14, "
                    "krylovdim 8, maxiter 3"}
    for prec in ("f64", "tf32x3"):
        t0 = time.perf_counter()
        d = dmrg.DMRG(n, 1.0, sb.Context(local), precision=prec)
        e, _ = d.run(sched, cutoff=1e-14, krylovdim=8, maxiter=3)
        out[prec] = {"energy": e, "seconds": time.perf_counter() - t0}
    exact = dmrg.exact_ground_energy(n, 1.0)
    out["exact"] = exact
    out["rel_diff_tf32x3_vs_f64"] = abs(out["tf32x3"]["energy"] - out["f64"]["energy"]) / abs(out["f64"]["energy"])
    out["rel_err_f64_vs_exact"] = abs(out["f64"]["energy"] - exact) / abs(exact)
    return out


# ── the CPU baseline: restatements of the reference path (numpy oracle, C++) ──

def cpu_matvec_rate(layout, host, budget_s: float, max_runs: int, keep=None):
    """Whole H_eff matvecs of the numpy oracle on the uniform reference blocks:
    (matvecs per second, matvecs, seconds)."""
    from oracle import sparse_oracle as so
    from sparsebackends_b200 import qn
    t = {}
    for name, (keys, data) in host.items():
        t[name] = so.BS(layout.dims[name], layout.n2[name], keys, list(range(1, len(keys) + 1)), data)
    lab = layout.labels

    def one():
        tt = dict(t)
        for c, a, b in qn.HeffChain.STEPS:
            tt[c] = so.contract(so.BS.empty(layout.dims[c], layout.n2[c]), lab[c], tt[a], lab[a], tt[b], lab[b])
        return tt["T4"]

    runs, start = 0, time.perf_counter()
    while runs < max_runs:
        t4 = one()
        runs += 1
        if time.perf_counter() - start > budget_s:
            break
    el = time.perf_counter() - start
    if keep is not None:
        keep.append(t4)
    return runs / el, runs, el


def cpp_matvec_rate(layout, host, budget_s: float, max_runs: int, keep=None):
    """``cpu_matvec_rate`` on the C++ restatement of contract_shared!
    (``oracle/cpu_ref``: compiled loops, one OpenBLAS dgemm per block pair, as
    the reference's mul!), operands resident on the C++ side."""
    from oracle import cpu_ref
    from sparsebackends_b200 import qn
    cpu_ref.build()
    t = {n: cpu_ref.Tensor(layout.dims[n], layout.n2[n], keys, data) for n, (keys, data) in host.items()}
    lab = layout.labels

    def one():
        tt = dict(t)
        for c, a, b in qn.HeffChain.STEPS:
            tt[c] = cpu_ref.contract(layout.dims[c], layout.n2[c], lab[c], tt[a], lab[a], tt[b], lab[b])
        return tt["T4"]

    runs, start = 0, time.perf_counter()
    while runs < max_runs:
        t4 = one()
        runs += 1
        if time.perf_counter() - start > budget_s:
            break
    el = time.perf_counter() - start
    if keep is not None:
        keep.append(t4)
    return runs / el, runs, el


def blas_threads():
    try:
        from threadpoolctl import threadpool_info
        th = [i.get("num_threads", 0) for i in threadpool_info() if i.get("user_api") == "blas"]
        return max(th) if th else os.cpu_count()
    except Exception:
        return os.cpu_count()


# ── main ──────────────────────────────────────────────────────────────────

def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def reduce_max(x: float, world: int) -> float:
    """Max over ranks (device time of the slowest replica)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_rate(world: int, steps: int, ms_max: float) -> float:
    """Whole-job matvec/s of `world` independent replicas that each ran
    `steps` matvecs, timed by the slowest one (ms_max)."""
    return world * steps / (ms_max / 1e3)


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def run_reference(args, world, rank):
    if rank != 0:
        return
    layout = workload(args.chi)
    host = host_tensors(layout, args.seed)
    # bounded sample: whole matvecs, warm-up capped at 1, timed steps capped by budget
    from sparsebackends_b200 import qn
    flops = qn.chain_flops(layout, padded=False)
    if args.warmup > 0:
        cpp_matvec_rate(layout, host, 0.0, 1)
    rate, runs, el = cpp_matvec_rate(layout, host, args.cpu_budget_s, max(1, args.steps))
    line = {
        "metric": METRIC, "value": rate, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
        "steps": runs, "steps_requested": args.steps, "warmup": min(args.warmup, 1), "ms_per_step": 1e3 / rate,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"two-site H_eff matvec, U(1) chi={args.chi}, MPO w=38 (J1-J2 6x6 sized)",
                   "chi": args.chi, "sectors": layout.left.dims, "mpo_channels": layout.mpo.dims,
                   "l2": "inputs larger than L2"},
        "gflops_algorithmic": flops * rate / 1e9,
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": blas_threads(), "kind": "port",
                         "sample": f"{runs} full matvec(s) of the same chi={args.chi} workload, C++ restatement "
                                   f"of contract_bs_bs.jl contract_shared! (g++ -O3, OpenBLAS 0.3.30 dgemm per "
                                   f"block pair)"},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args, world, rank, local):
    import ctypes as C
    import torch
    import sparsebackends_b200 as sb
    from sparsebackends_b200 import qn

    torch.cuda.set_device(local)
    layout = workload(args.chi)
    host, host_r = host_tensors(layout, args.seed, with_ragged=True)
    ctx = sb.Context(local)
    # ragged (unpadded sectors): the headline form; uniform: the reference layout
    dev_r = {n: sb.NewBlockSparseSorted(layout.dims[n], layout.n2[n], k, None, d, ctx=ctx, block_dims=e)
             for n, (k, d, e) in host_r.items()}
    dev_u = {n: sb.NewBlockSparseSorted(layout.dims[n], layout.n2[n], k, None, d, ctx=ctx) for n, (k, d) in host.items()}
    chain_r, chain_u = qn.HeffChain(layout, ctx), qn.HeffChain(layout, ctx)
    # the same matvec associated as psi·L·(W1·W2)·R (W12 recomputed every step)
    chain_w = qn.HeffChain(layout, ctx, w12=True)
    stream = torch.cuda.ExternalStream(ctx.stream)
    flops_alg = qn.chain_flops(layout, padded=False)
    flops_pad = qn.chain_flops(layout, padded=True)
    flops_w = qn.chain_flops(layout, padded=False, steps=qn.HeffChain.STEPS_W12)

    def apply_r():
        return chain_r.apply(dev_r["psi"], dev_r["L"], dev_r["W1"], dev_r["W2"], dev_r["R"])

    def apply_u():
        return chain_u.apply(dev_u["psi"], dev_u["L"], dev_u["W1"], dev_u["W2"], dev_u["R"])

    def apply_w():
        return chain_w.apply(dev_r["psi"], dev_r["L"], dev_r["W1"], dev_r["W2"], dev_r["R"])

    for _ in range(max(args.warmup, 3)):
        apply_r()
        apply_u()
        apply_w()
    ctx.synchronize()
    d_w, d_r4 = chain_w.out["T4"].data, chain_r.out["T4"].data
    agree_w = float(np.linalg.norm(d_w - d_r4) / max(np.linalg.norm(d_r4), 1e-300))
    assert chain_w.out["T4"].keys == chain_r.out["T4"].keys and agree_w < 1e-12, agree_w
    # the two forms agree (same keys; unpadded blocks equal the padded result)
    ur, uu = sb.to_uniform(chain_r.out["T4"]), chain_u.out["T4"]
    assert ur.keys == uu.keys
    d_r, d_u = ur.data, uu.data
    agree = float(np.linalg.norm(d_r - d_u) / max(np.linalg.norm(d_u), 1e-300))
    assert agree < 1e-12, agree
    peak = fp64_peak_tflops() if rank == 0 else 0.0
    torch.cuda.synchronize()

    def timed(fn, steps, profile=False):
        barrier(world)
        ctx.synchronize()
        if profile:
            ctx.set_profiling(True)
        l0 = ctx.launch_count
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        for _ in range(steps):
            fn()
        e.record(stream)
        ctx.synchronize()
        prof = {k: ctx.profile(k) for k in ("gemm", "gemm_thin", "permute", "outer", "axpy")} if profile else None
        if profile:
            ctx.set_profiling(False)
        barrier(world)
        return reduce_max(s.elapsed_time(e), world), ctx.launch_count - l0, prof

    # ── device-resident throughput (value): ragged form ──
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    ms, launches, _ = timed(apply_r, args.steps)
    clocks = sampler.stop()
    # per-kernel CUDA-event times (roofline, kernel shares) from a second,
    # profiled pass: the event records are kept out of the timed steps above
    _, _, prof = timed(apply_r, args.steps, profile=True)
    value = replica_rate(world, args.steps, ms)
    # uniform (reference layout) for comparison
    ms_u, _, _ = timed(apply_u, args.steps)
    _, _, prof_u = timed(apply_u, args.steps, profile=True)
    value_u = replica_rate(world, args.steps, ms_u)
    # the reference layout without cropping its zero padding (a context with
    # SPARSEB_AUTO_CROP=0: every block GEMM runs on the padded extents)
    saved = os.environ.get("SPARSEB_AUTO_CROP")
    os.environ["SPARSEB_AUTO_CROP"] = "0"
    try:
        ctx_nc = sb.Context(local)
    finally:
        if saved is None:
            os.environ.pop("SPARSEB_AUTO_CROP", None)
        else:
            os.environ["SPARSEB_AUTO_CROP"] = saved
    dev_nc = {n: sb.NewBlockSparseSorted(layout.dims[n], layout.n2[n], k, None, d, ctx=ctx_nc)
              for n, (k, d) in host.items()}
    chain_nc = qn.HeffChain(layout, ctx_nc)
    stream_nc = torch.cuda.ExternalStream(ctx_nc.stream)

    def apply_nc():
        return chain_nc.apply(dev_nc["psi"], dev_nc["L"], dev_nc["W1"], dev_nc["W2"], dev_nc["R"])

    for _ in range(2):
        apply_nc()
    barrier(world)
    ctx_nc.synchronize()
    s_nc, e_nc = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s_nc.record(stream_nc)
    for _ in range(args.steps):
        apply_nc()
    e_nc.record(stream_nc)
    ctx_nc.synchronize()
    barrier(world)
    ms_nc = reduce_max(s_nc.elapsed_time(e_nc), world)
    nc_diff = float(np.linalg.norm(chain_nc.out["T4"].data - chain_u.out["T4"].data) /
                    max(np.linalg.norm(chain_nc.out["T4"].data), 1e-300))
    assert nc_diff < 1e-12, nc_diff
    del chain_nc, dev_nc
    value_nc = replica_rate(world, args.steps, ms_nc)
    # the W12 association
    ms_w, _, _ = timed(apply_w, args.steps)
    _, _, prof_w = timed(apply_w, args.steps, profile=True)
    value_w = replica_rate(world, args.steps, ms_w)

    # ── the FP64 chain with the tile shapes picked by the autotuner
    # (SPARSEB_AUTOTUNE=1, read at context creation; off by default)
    os.environ["SPARSEB_AUTOTUNE"] = "1"
    ctx_at = sb.Context(local)
    del os.environ["SPARSEB_AUTOTUNE"]
    dev_at = {n: sb.NewBlockSparseSorted(layout.dims[n], layout.n2[n], k, None, d, ctx=ctx_at, block_dims=e)
              for n, (k, d, e) in host_r.items()}
    chain_at = qn.HeffChain(layout, ctx_at)
    stream_at = torch.cuda.ExternalStream(ctx_at.stream)
    for _ in range(max(args.warmup, 3)):  # the first apply tunes each contraction
        chain_at.apply(dev_at["psi"], dev_at["L"], dev_at["W1"], dev_at["W2"], dev_at["R"])
    barrier(world)
    ctx_at.synchronize()
    s_at, e_at = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s_at.record(stream_at)
    for _ in range(args.steps):
        chain_at.apply(dev_at["psi"], dev_at["L"], dev_at["W1"], dev_at["W2"], dev_at["R"])
    e_at.record(stream_at)
    ctx_at.synchronize()
    barrier(world)
    ms_at = reduce_max(s_at.elapsed_time(e_at), world)
    at_diff = float(np.linalg.norm(chain_at.out["T4"].data - chain_r.out["T4"].data) /
                    max(np.linalg.norm(chain_r.out["T4"].data), 1e-300))
    autotuned = {"value": replica_rate(world, args.steps, ms_at), "unit": UNIT, "ms_per_step": ms_at / args.steps,
                 "rel_diff_vs_headline": at_diff,
                 "note": "SPARSEB_AUTOTUNE=1: the first launch of each block-shape histogram times the heuristic's "
                         "tile choice against every tile shape on its own operands and keeps the fastest"}
    del chain_at, dev_at

    # ── mixed precision: the tiled steps on the tcgen05 tensor cores (3xTF32),
    # FP32-stored intermediates, in both associations of the chain
    ctx_mx = sb.Context(local)
    ctx_mx.set_precision("tf32x3")
    dev_mx = {n: sb.NewBlockSparseSorted(layout.dims[n], layout.n2[n], k, None, d, ctx=ctx_mx, block_dims=e)
              for n, (k, d, e) in host_r.items()}
    stream_mx = torch.cuda.ExternalStream(ctx_mx.stream)
    mixed = {}
    for name, w12 in (("psi_L_W1_W2_R", False), ("w12", True)):
        ch = qn.HeffChain(layout, ctx_mx, w12=w12, f32_intermediates=True)
        def fn(c=ch):
            # a new psi every step, as in Lanczos: its packed operand images are
            # rebuilt (L and R keep theirs)
            sb.scale_(dev_mx["psi"], 1.0)
            return c.apply(dev_mx["psi"], dev_mx["L"], dev_mx["W1"], dev_mx["W2"], dev_mx["R"])
        for _ in range(max(args.warmup, 3)):
            fn()
        barrier(world)
        ctx_mx.synchronize()
        s_m, e_m = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s_m.record(stream_mx)
        for _ in range(args.steps):
            fn()
        e_m.record(stream_mx)
        ctx_mx.synchronize()
        barrier(world)
        ms_m = reduce_max(s_m.elapsed_time(e_m), world)
        ctx_mx.set_profiling(True)
        for _ in range(args.steps):
            fn()
        ctx_mx.synchronize()
        pm = {k: ctx_mx.profile(k) for k in ("gemm_tc", "gemm_thin", "other")}
        ctx_mx.set_profiling(False)
        ref_d = chain_r.out["T4"].data
        got_d = ch.out["T4"].data
        gb, rb = ch.out["T4"].blocks_by_key(), chain_r.out["T4"].blocks_by_key()
        blk_err = max(float(np.linalg.norm(gb[k] - v) / max(np.linalg.norm(v), 1e-300)) for k, v in rb.items())
        mixed[name] = {"value": replica_rate(world, args.steps, ms_m), "ms_per_step": ms_m / args.steps,
                       "rel_err_vs_fp64": float(np.linalg.norm(got_d - ref_d) / np.linalg.norm(ref_d)),
                       "max_block_rel_err_vs_fp64": blk_err,
                       "kernel_ms_per_step": {k: v["ms"] / args.steps for k, v in pm.items()},
                       "prof": pm}
        del ch

    # ── end to end through the public API (pinned host psi in, H·psi out) ──
    lib = ctx._lib

    def make_e2e(ragged):
        keys = host_r["psi"][0] if ragged else host["psi"][0]
        data = host_r["psi"][1] if ragged else host["psi"][1]
        exts = host_r["psi"][2]
        pin_in = torch.empty(max(data.size, 1), dtype=torch.float64, pin_memory=True)
        pin_in.numpy()[: data.size] = data
        chain = chain_r if ragged else chain_u
        out_len = chain.out["T4"]._layout()[2]
        pin_out = torch.empty(max(out_len, 1), dtype=torch.float64, pin_memory=True)
        in_ptr = C.cast(C.c_void_p(pin_in.data_ptr()), C.POINTER(C.c_double))
        out_ptr = C.cast(C.c_void_p(pin_out.data_ptr()), C.POINTER(C.c_double))
        dims = layout.dims["psi"]
        kflat = sb._i64([x for k in keys for x in k])
        bflat = sb._i64([x for e in exts for x in e])
        devs = dev_r if ragged else dev_u

        def once():
            p = sb.NewBlockSparseSorted.__new__(sb.NewBlockSparseSorted)
            h = C.c_void_p()
            if ragged:
                st = lib.sb_tensor_create_bs_ragged(ctx._h, len(dims), sb._i64(dims), layout.n2["psi"], len(keys),
                                                    kflat, bflat, in_ptr, C.byref(h))
            else:
                st = lib.sb_tensor_create_bs(ctx._h, len(dims), sb._i64(dims), layout.n2["psi"], len(keys), kflat,
                                             None, in_ptr, C.byref(h))
            sb._check(ctx, st)
            sb._Tensor.__init__(p, ctx, h)
            out = chain.apply(p, devs["L"], devs["W1"], devs["W2"], devs["R"])
            sb._check(ctx, lib.sb_tensor_export_bs(ctx._h, out._h, None, None, out_ptr))

        return once, int(data.size * 8), int(out_len * 8)

    e2e_r, h2d_r, d2h_r = make_e2e(True)
    e2e_u, h2d_u, d2h_u = make_e2e(False)
    for _ in range(2):
        e2e_r()
        e2e_u()
    ms_e2e, _, _ = timed(e2e_r, args.steps)
    ms_e2e_u, _, _ = timed(e2e_u, args.steps)
    e2e_serial = replica_rate(world, args.steps, ms_e2e)
    e2e_value_u = replica_rate(world, args.steps, ms_e2e_u)

    # ── end to end, two requests in flight (serving loop): two contexts with
    # their own streams and operator copies; request i runs on slot i % 2, so
    # the host<->device copies of one request overlap the kernels of the other.
    # The kernels of the two requests do not overlap: each apply waits for the
    # previous request's apply (an event), as two chains sharing the SMs and L2
    # ran slower (191.5 against 204.9 matvec/s at chi=2048).
    ctx2 = sb.Context(local)
    dev_r2 = {n: sb.NewBlockSparseSorted(layout.dims[n], layout.n2[n], k, None, d, ctx=ctx2, block_dims=e)
              for n, (k, d, e) in host_r.items()}
    pkeys, pdata, pexts = host_r["psi"]
    out_len = chain_r.out["T4"]._layout()[2]
    kflat = sb._i64([x for k in pkeys for x in k])
    bflat = sb._i64([x for e in pexts for x in e])
    dims_psi = sb._i64(layout.dims["psi"])

    class Slot:
        def __init__(self, c, devs):
            self.ctx, self.devs, self.chain = c, devs, qn.HeffChain(layout, c)
            self.pin_in = torch.empty(max(pdata.size, 1), dtype=torch.float64, pin_memory=True)
            self.pin_in.numpy()[: pdata.size] = pdata
            self.pin_out = torch.empty(max(out_len, 1), dtype=torch.float64, pin_memory=True)
            self.in_ptr = C.cast(C.c_void_p(self.pin_in.data_ptr()), C.POINTER(C.c_double))
            self.out_ptr = C.cast(C.c_void_p(self.pin_out.data_ptr()), C.POINTER(C.c_double))
            self.psi = None
            self.stream = torch.cuda.ExternalStream(c.stream)
            self.applied = torch.cuda.Event()

        def step(self, after):
            c = self.ctx
            h = C.c_void_p()
            sb._check(c, lib.sb_tensor_create_bs_ragged(c._h, len(layout.dims["psi"]), dims_psi, layout.n2["psi"],
                                                        len(pkeys), kflat, bflat, self.in_ptr, C.byref(h)))
            p = sb.NewBlockSparseSorted.__new__(sb.NewBlockSparseSorted)
            sb._Tensor.__init__(p, c, h)
            self.psi = p  # released on this slot's stream at its next request
            if after is not None:
                self.stream.wait_event(after)
            out = self.chain.apply(p, self.devs["L"], self.devs["W1"], self.devs["W2"], self.devs["R"])
            self.applied.record(self.stream)
            sb._check(c, lib.sb_tensor_export_bs_async(c._h, out._h, None, None, self.out_ptr))
            return self.applied

    slots = [Slot(ctx, dev_r), Slot(ctx2, dev_r2)]
    s1, s2 = stream, torch.cuda.ExternalStream(ctx2.stream)

    def timed_pipelined(steps):
        barrier(world)
        ctx.synchronize()
        ctx2.synchronize()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(s1)
        s2.wait_event(start)
        after = None
        for i in range(steps):
            after = slots[i % 2].step(after)
        done2 = torch.cuda.Event()
        done2.record(s2)
        s1.wait_event(done2)
        end.record(s1)
        ctx.synchronize()
        ctx2.synchronize()
        barrier(world)
        return reduce_max(start.elapsed_time(end), world)

    timed_pipelined(4)
    ms_pipe = timed_pipelined(args.steps)
    e2e_value = replica_rate(world, args.steps, ms_pipe)
    for sl in slots:  # every request returned H·psi (deterministic kernels: bit-exact)
        assert np.array_equal(sl.pin_out.numpy()[:out_len], chain_r.out["T4"].data)

    # ── the same matvec replayed as one CUDA graph (host planning paid once),
    # at chi=2048 and at a small bond dimension where host work would dominate
    chain_g = qn.HeffChain(layout, ctx)
    graph = chain_g.capture(dev_r["psi"], dev_r["L"], dev_r["W1"], dev_r["W2"], dev_r["R"])
    for _ in range(3):
        graph.launch()
    ms_g, _, _ = timed(graph.launch, args.steps)
    assert np.array_equal(chain_g.out["T4"].data, chain_r.out["T4"].data)

    def small_chi_rates(chi_s, steps):
        lay_s = workload(chi_s)
        _, hr = host_tensors(lay_s, args.seed, with_ragged=True)
        ds = {n: sb.NewBlockSparseSorted(lay_s.dims[n], lay_s.n2[n], k, None, d, ctx=ctx, block_dims=e)
              for n, (k, d, e) in hr.items()}
        ch = qn.HeffChain(lay_s, ctx)
        args_s = (ds["psi"], ds["L"], ds["W1"], ds["W2"], ds["R"])
        for _ in range(3):
            ch.apply(*args_s)
        ms_e, _, _ = timed(lambda: ch.apply(*args_s), steps)
        chg = qn.HeffChain(lay_s, ctx)
        gs = chg.capture(*args_s)
        for _ in range(3):
            gs.launch()
        ms_s, _, _ = timed(gs.launch, steps)
        assert np.array_equal(chg.out["T4"].data, ch.out["T4"].data)
        return {"chi": chi_s, "eager_matvec_per_s": replica_rate(world, steps, ms_e),
                "graph_matvec_per_s": replica_rate(world, steps, ms_s)}

    def centre_problem_leg(steps):
        """The two-site H_eff at the centre bond of a canonical Heisenberg MPS
        (N = 16, chi = 64, centre link {4, 12, 32, 12, 4}): the reference's
        plain FP64 CPU matvec case, eager and replayed from a graph, against the
        oracle's chain on the zero-padded operands."""
        from sparsebackends_b200 import dmrg
        lay1, psi1, L1, W1_, R1 = dmrg.canonical_center_problem(ctx)
        a1 = (psi1, L1, W1_, W1_, R1)
        ch = qn.HeffChain(lay1, ctx)
        for _ in range(3):
            ch.apply(*a1)
        ms_e, _, _ = timed(lambda: ch.apply(*a1), steps)
        chg = qn.HeffChain(lay1, ctx)
        g1 = chg.capture(*a1)
        for _ in range(3):
            g1.launch()
        ms_s, _, _ = timed(g1.launch, steps)
        assert np.array_equal(chg.out["T4"].data, ch.out["T4"].data)
        out = {"workload": "two-site H_eff matvec at the centre bond of a canonical Heisenberg MPS, N=16, "
                           "chi=64 (centre link 2Sz=-4..4 at {4,12,32,12,4}; psi on links {8,22,22,8}), MPO w=5",
               "eager_matvec_per_s": replica_rate(world, steps, ms_e),
               "graph_matvec_per_s": replica_rate(world, steps, ms_s),
               "gflop_per_matvec_algorithmic": qn.chain_flops(lay1, padded=False) / 1e9,
               "l2": "inputs L2-resident (a few MB)"}
        if rank == 0 and world == 1 and not args.no_cpu_baseline:
            host1 = {}
            for name, t in (("psi", psi1), ("L", L1), ("W1", W1_), ("W2", W1_), ("R", R1)):
                u = sb.to_uniform(t)
                host1[name] = (u.keys, np.array(u.data, copy=True))
            last = []
            cpu_matvec_rate(lay1, host1, 0.0, 1, keep=last)  # the oracle's result, for the check below
            rate, runs, el = cpp_matvec_rate(lay1, host1, 5.0, 4000)
            got = sb.to_uniform(ch.out["T4"])
            ref = last[-1]
            assert got.keys == ref.keys
            gb = got.blocks_by_key()
            out["max_block_rel_err_vs_oracle"] = max(
                float(np.linalg.norm(np.asarray(gb[k]) - v) / max(np.linalg.norm(v), 1e-300))
                for k, v in ref.blocks_by_key().items())
            out["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": blas_threads(), "kind": "port",
                                   "sample": f"{runs} matvecs in {el:.1f} s, C++ restatement of contract_shared! "
                                             f"(g++ -O3, OpenBLAS dgemm per block pair) on the uniform blocks"}
        return out

    centre_leg = centre_problem_leg(max(200, args.steps))

    graph_leg = {"value": replica_rate(world, args.steps, ms_g), "unit": UNIT,
                 "note": "the H_eff chain captured once (sb_ctx_capture_begin/end) and replayed with sb_graph_launch",
                 "small_chi": small_chi_rates(256, 200)}

    # ── one Lanczos eigensolve as DMRG calls it (krylovdim 3, maxiter 1) ──
    from sparsebackends_b200 import krylov
    op = qn.HeffOperator(layout, dev_r["L"], dev_r["W1"], dev_r["W2"], dev_r["R"], ctx)
    krylov.eigsolve(op, dev_r["psi"], 1, "SR", krylovdim=3, maxiter=1, tol=1e-14)
    ctx.synchronize()
    t0 = time.perf_counter()
    nsolve = max(2, min(5, args.steps // 10))
    for _ in range(nsolve):
        krylov.eigsolve(op, dev_r["psi"], 1, "SR", krylovdim=3, maxiter=1, tol=1e-14)
    ctx.synchronize()
    ms_solve = (time.perf_counter() - t0) * 1e3 / nsolve
    lanczos = {"ms_per_solve": ms_solve, "matvecs_per_solve": 3, "matvec_ms": ms / args.steps,
               "vector_ops_and_sync_ms": ms_solve - 3 * ms / args.steps,
               "note": "wall time of eigsolve(krylovdim=3, maxiter=1) on the device vectors; dot/norm results "
                       "return to the host, as KrylovKit's scalars do"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, runs, el = cpp_matvec_rate(layout, host, args.cpu_budget_s, 8)
        cpu = {"value": rate, "unit": UNIT, "cores": blas_threads(), "kind": "port",
               "sample": f"{runs} full matvec(s) of the same workload in {el:.1f} s, C++ restatement of "
                         f"contract_shared! (contract_bs_bs.jl:572-730; g++ -O3, one OpenBLAS 0.3.30 dgemm per "
                         f"block pair as the reference's mul!) on the reference's uniform (zero-padded) blocks"}

    if rank != 0:
        return
    tf32_peak = tf32_peak_tflops()
    mx_energy = mixed_dmrg_energy(local)
    tcp = mixed["w12"]["prof"]["gemm_tc"]
    tc_alg = tcp["flops"] / (tcp["ms"] * 1e-3) / 1e12 if tcp["ms"] > 0 else 0.0
    for m in mixed.values():
        m.pop("prof")
    mixed_line = {
        "value": mixed["w12"]["value"], "unit": UNIT,
        "form": "block GEMMs of psi*L and R*T3 on tcgen05 in 3xTF32 (TF32 hi/lo split of every operand, FP32 "
                "accumulation in Kahan-summed chunks), MPO steps in FP64 arithmetic on FP32-stored intermediates; "
                "association psi*L*(W1*W2)*R; Lanczos vectors, inner products and norms FP64",
        "dtype": "tf32x3",
        "ratio_vs_plain_fp64": mixed["w12"]["value"] / value,
        "ratio_vs_plain_fp64_same_association": mixed["w12"]["value"] / value_w,
        "forms": mixed,
        "roofline": {"bound": "tensor", "kernel": "k_gemm_tc (tcgen05.mma kind::tf32, 128xN tiles, warp-specialized)",
                     "achieved_tf32_ops": 3.0 * tc_alg, "peak": tf32_peak, "unit": "TFLOP/s",
                     "frac": 3.0 * tc_alg / tf32_peak if tf32_peak else None,
                     "achieved_algorithmic": tc_alg,
                     "note": "three TF32 products per FP64 multiply-add (3xTF32); peak measured live: torch.matmul "
                             "float32 with TF32 allowed, 8192^3, best of 10",
                     "launches": tcp["launches"], "kernel_ms_per_step": tcp["ms"] / args.steps},
        "dmrg_energy": mx_energy,
    }
    g = prof["gemm"]
    achieved = g["flops"] / (g["ms"] * 1e-3) / 1e12 if g["ms"] > 0 else 0.0
    th = prof["gemm_thin"]
    thin_gbs = th["bytes"] / (th["ms"] * 1e-3) / 1e9 if th["ms"] > 0 else 0.0
    hbm_peak = measured_hbm_gbs()
    gu, gtu = prof_u["gemm"], prof_u["gemm_thin"]
    permute = permute_stage(ctx, dev_u["L"], hbm_peak)
    # single-GPU studies: measured at N = 1 only, so that a replica run does not
    # hold every GPU while rank 0 alone runs them
    serving = serving_leg(args.seed) if world == 1 else None
    pxp_line = pxp_leg(local, args.steps) if world == 1 else None
    j1j2_line = j1j2_leg(local, 2048, 60.0, "gram") if world == 1 else None
    # the vendor library on the same block lists, after every timed leg (its
    # many small launches stay out of the launch lists profiled from this run)
    library = cublas_block_lists(layout)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": max(args.warmup, 3), "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"two-site H_eff matvec, U(1) chi={args.chi}, MPO w=38 (J1-J2 6x6 sized)",
                   "chi": args.chi, "sectors": layout.left.dims, "mpo_channels": layout.mpo.dims,
                   "format": "ragged block extents (unpadded U(1) sectors); uniform reference layout reported "
                             "in uniform_format",
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                   "l2": "inputs larger than L2 (operators ~0.6 GB, intermediates ~2.3 GB each)"},
        "gflops_algorithmic": flops_alg * value / 1e9,
        "roofline": {"bound": "tensor", "kernel": "k_gemm_f64_edges (DMMA m8n8k4, 64x64 tiles with 64x32 / 64x48 / "
                                                       "32x64 / 48x64 edge tiles; steps psi*L and R*T3)",
                     "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak if peak else None,
                     "peak_source": "measured live: torch.matmul float64 8192^3, best of 10 (cuBLAS DGEMM)",
                     "flops_per_launch": g["flops"] / max(g["launches"], 1),
                     "traffic": traffic_per_launch(args.chi, "k_gemm_f64"), "launches": g["launches"],
                     "kernel_ms_per_step": g["ms"] / args.steps},
        "roofline_mpo_steps": {"bound": "hbm", "kernel": "k_gemm_thin_p (steps T1*W1 and T2*W2, K <= 16)",
                               "achieved": thin_gbs, "peak": hbm_peak, "unit": "GB/s",
                               "frac": thin_gbs / hbm_peak if hbm_peak else None,
                               "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)",
                               "bytes_per_launch": th["bytes"] / max(th["launches"], 1),
                               "traffic": traffic_per_launch(args.chi, "k_gemm_thin"), "launches": th["launches"],
                               "kernel_ms_per_step": th["ms"] / args.steps},
        "kernel_time_share": {k: v["ms"] / max(1e-9, sum(x["ms"] for x in prof.values())) for k, v in prof.items()},
        "library_baseline": library,
        "permute_stage": permute,
        "serving": serving,
        "pxp_chain": pxp_line,
        "j1j2_cylinder_dmrg": j1j2_line,
        "uniform_format": {"value": value_u, "ms_per_step": ms_u / args.steps,
                           "note": "contract! on the reference's zero-padded blocks; psi*L and R*T3 crop the padding "
                                   "inside contract_shared! (scan, harmonised extents, ragged GEMM, padded result)",
                           "gflops_executed": (gu["flops"] + gtu["flops"]) / args.steps * value_u / 1e9,
                           "gemm_tflops": (gu["flops"] + gtu["flops"]) / ((gu["ms"] + gtu["ms"]) * 1e-3) / 1e12
                           if gu["ms"] + gtu["ms"] > 0 else 0.0,
                           "e2e": {"value": e2e_value_u, "unit": UNIT, "h2d_bytes_per_step": h2d_u,
                                   "d2h_bytes_per_step": d2h_u},
                           "no_crop": {"value": value_nc, "ms_per_step": ms_nc / args.steps,
                                       "gflops_executed": flops_pad * value_nc / 1e9,
                                       "rel_diff_vs_cropped": nc_diff,
                                       "note": "SPARSEB_AUTO_CROP=0: every block GEMM on the padded extents"}},
        "ragged_vs_uniform_rel_diff": agree,
        "autotuned": autotuned,
        "w12_association": {"value": value_w, "unit": UNIT, "ms_per_step": ms_w / args.steps,
                            "steps": "W12 = W1*W2, T1 = psi*L, T3 = T1*W12, T4 = R*T3 (four contract! calls, "
                                     "W12 recomputed every step; the headline runs ITensorMPS's order psi*L, *W1, "
                                     "*W2, *R)",
                            "gflops_algorithmic": flops_w * value_w / 1e9,
                            "mpo_step_ms": prof_w["gemm_thin"]["ms"] / args.steps,
                            "rel_diff_vs_reference_order": agree_w},
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d_r, "d2h_bytes_per_step": d2h_r,
                "mode": "two requests in flight (two contexts/streams; copies overlap the other request's "
                        "kernels, the kernels of the two run one request after the other); every request "
                        "uploads psi from pinned host memory and reads H*psi back",
                "serial": {"value": e2e_serial, "unit": UNIT,
                           "mode": "one request at a time: upload, apply, blocking read-back"}},
        "lanczos": lanczos,
        "mixed_precision": mixed_line,
        "graph_replay": graph_leg,
        "centre_bond_n16_chi64": centre_leg,
        "gpu_launches": launches,
        "clocks": clocks,
    }
    print(json.dumps(line), flush=True)


def pxp_leg(local: int, steps: int, cpu_budget_s: float = 0.0, seed: int = 64):
    """The PXP chain (N = 64, chi = 256, MPO bond 4 in COO): the two-site
    H_eff matvec in plain FP64 and with its two dense contractions in 3xTF32
    (error of the 3xTF32 result against the FP64 one), and the MPO x MPS apply
    on every site tensor (COO x block-sparse scaled adds).  With
    ``cpu_budget_s`` > 0 the oracle port runs the same matvec on the host
    cores beside it."""
    import torch
    import sparsebackends_b200 as sb
    from sparsebackends_b200 import pxp
    torch.cuda.set_device(local)
    ctx = sb.Context(local)
    t0 = time.perf_counter()
    prob = pxp.PxpProblem(64, 256, seed, ctx=ctx)
    ctx.synchronize()
    setup_s = time.perf_counter() - t0
    stream = torch.cuda.ExternalStream(ctx.stream)
    dims = pxp.bond_dims(prob.n, prob.chi)
    dl, dr = dims[prob.c - 1], dims[prob.c + 1]
    # T1 = L*psi: 4 channels x 4 (s1, s2) blocks of dl x dl x dr; T4 = T3*R:
    # 16 (s1', s2', wr) products of dl x dr x dr
    nl, nr = len(prob.L.keys), len(prob.R.keys)
    flops = 2.0 * (nl * 4 * dl * dl * dr + 4 * nr * dl * dr * dr)

    def timed(fn, n):
        for _ in range(3):
            fn()
        ctx.synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        for _ in range(n):
            fn()
        e.record(stream)
        ctx.synchronize()
        return s.elapsed_time(e) / n

    kinds = ("gemm", "gemm_thin", "gemm_tc", "tc_pack", "permute", "outer", "axpy", "vector", "other")

    def forms():
        """eager ms, graph-replay ms and per-kind kernel ms of one matvec"""
        out = prob.apply(prob.psi)
        ms = timed(lambda: prob.apply(prob.psi), steps)
        ctx.set_profiling(True)
        for _ in range(5):
            prob.apply(prob.psi)
        ctx.synchronize()
        kern = {k: ctx.profile(k)["ms"] / 5 for k in kinds}
        ctx.set_profiling(False)
        graph, gout = prob.capture(prob.psi)
        ms_g = timed(graph.launch, steps)
        del graph, gout
        return out, ms, ms_g, {k: v for k, v in kern.items() if v > 0}

    out64, ms64, ms64g, kern64 = forms()
    ctx.set_precision("tf32x3")
    try:
        out32, ms32, ms32g, kern32 = forms()
    finally:
        ctx.set_precision("f64")
    ops = prob.aliased_operands()
    psi_d = sb.DenseTensor(prob.psi_host, ctx=ctx)
    ms_al = timed(lambda: prob.apply_aliased(psi_d, ops), steps)
    b64, b32 = out64.blocks_by_key(), out32.blocks_by_key()
    scale = max(float(np.max(np.abs(v))) for v in b64.values())
    err = max(float(np.max(np.abs(b32[k] - v))) for k, v in b64.items()) / scale
    sites = [prob._bs(*pxp.site_blocks(a)) for a in prob.sites if a is not None]
    site_bytes = sum(8 * a.size for a in prob.sites if a is not None)
    outs = [prob.apply_mpo(a) for a in sites]
    out_bytes = sum(8 * len(o.keys) * o.blksize for o in outs)
    ms_mpo = timed(lambda: [prob.apply_mpo(a) for a in sites], max(3, steps // 10))
    res = {"workload": "PXP chain N=64, OBC, no U(1); MPO bond 4 (8 nonzeros) in COO; random MPS chi=256; "
                       "two-site H_eff at the centre (sites 32, 33), environments built on the device",
           "setup_s": setup_s,
           "heff_fp64": {"value": 1e3 / ms64, "unit": "matvec/s", "ms": ms64, "gflops_algorithmic": flops / ms64 / 1e6,
                         "graph": {"value": 1e3 / ms64g, "ms": ms64g, "gflops_algorithmic": flops / ms64g / 1e6},
                         "kernel_ms": kern64},
           "heff_tf32x3": {"value": 1e3 / ms32, "unit": "matvec/s", "ms": ms32,
                           "gflops_algorithmic": flops / ms32 / 1e6,
                           "graph": {"value": 1e3 / ms32g, "ms": ms32g, "gflops_algorithmic": flops / ms32g / 1e6},
                           "kernel_ms": kern32,
                           "rel_err_vs_fp64": err,
                           "form": "psi*L and T3*R on tcgen05 in 3xTF32 (FP32 accumulation); the MPO steps are "
                                   "scaled adds by the exact 0/1 entries in FP64"},
           "heff_aliased_fp64": {"value": 1e3 / ms_al, "unit": "matvec/s", "ms": ms_al,
                                 "form": "W aliased (templates I, P, X), dense psi and environments: "
                                         "contract_shared! of the aliased backend, FP64 block GEMMs"},
           "mpo_apply": {"sites": len(sites), "ms_all_sites": ms_mpo, "sites_per_s": 1e3 * len(sites) / ms_mpo,
                         "gb_per_s_algorithmic": (site_bytes + out_bytes) / ms_mpo / 1e6,
                         "form": "COO x block-sparse (contract_prefix!), FP64"},
           "flops_per_matvec": flops}
    if cpu_budget_s > 0:
        from oracle import cpu_ref
        from oracle.pxp_oracle import OracleProblem
        ora = OracleProblem(64, 256, seed)
        cpu_ref.build()
        apply, x = cpu_ref.pxp_heff_runner(ora)
        n, t0 = 0, time.perf_counter()
        while n < 2 or (time.perf_counter() - t0 < cpu_budget_s and n < 2000):
            apply(x)
            n += 1
        el = time.perf_counter() - t0
        res["cpu_baseline"] = {"value": n / el, "unit": "matvec/s", "cores": blas_threads(), "kind": "port",
                               "sample": f"{n} matvecs in {el:.1f} s, C++ restatement (g++ -O3: contract_shared! "
                                         f"with OpenBLAS dgemm, fuse_two_axes!, contract_prefix! scaled adds)"}
    return res


def run_mixed_only(args, world, rank, local):
    """The 3xTF32 chain alone (W12 association, FP32 intermediates): warm-up
    and timed steps on the device-resident operands of ``workload(chi)``."""
    import torch
    import sparsebackends_b200 as sb
    from sparsebackends_b200 import qn
    torch.cuda.set_device(local)
    layout = workload(args.chi)
    _, host_r = host_tensors(layout, args.seed, with_ragged=True)
    ctx = sb.Context(local)
    ctx.set_precision("tf32x3")
    dev = {n: sb.NewBlockSparseSorted(layout.dims[n], layout.n2[n], k, None, d, ctx=ctx, block_dims=e)
           for n, (k, d, e) in host_r.items()}
    ch = qn.HeffChain(layout, ctx, w12=True, f32_intermediates=True)
    stream = torch.cuda.ExternalStream(ctx.stream)
    def step():
        sb.scale_(dev["psi"], 1.0)  # a new psi every step, as in Lanczos (its images are rebuilt)
        ch.apply(dev["psi"], dev["L"], dev["W1"], dev["W2"], dev["R"])

    for _ in range(max(args.warmup, 3)):
        step()
    barrier(world)
    ctx.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record(stream)
    for _ in range(args.steps):
        step()
    e.record(stream)
    ctx.synchronize()
    barrier(world)
    ms = reduce_max(s.elapsed_time(e), world)
    if rank == 0:
        print(json.dumps({"leg": "mixed", "chi": args.chi, "steps": args.steps, "ms_per_step": ms / args.steps,
                          "value": replica_rate(world, args.steps, ms), "unit": UNIT}), flush=True)


def run_dmrg_leg(args, world, rank, local):
    """Two-site DMRG of the Heisenberg chain (J = 1, open, U(1) 2Sz = 0) from
    the Neel state: 5 sweeps with maxdim 64, 128, 256, 512, 512, cutoff 1e-10,
    krylovdim 3, maxiter 1 per bond, in plain FP64 and in the 3xTF32 form (the
    H_eff applies on the tensor cores, FP64 Rayleigh-quotient energies).  Every
    step runs on the device (contractions, Lanczos vector operations, the SVD
    per centre charge); the host holds keys, the tridiagonal eigenproblem and
    the singular values for the truncation."""
    import torch
    import sparsebackends_b200 as sb
    from sparsebackends_b200 import dmrg
    torch.cuda.set_device(local)
    kinds = ("gemm", "gemm_thin", "gemm_tc", "tc_pack", "permute", "outer", "axpy", "vector", "other")

    def run(sched, krylovdim, maxiter):
        out = {}
        for prec in ("f64", "tf32x3"):
            ctx = sb.Context(local)
            d = dmrg.DMRG(args.dmrg_n, 1.0, ctx, precision=prec, device_split=True)  # no host linear algebra
            ctx.set_profiling(True)
            energies, secs = [], []
            for m in sched:
                t0 = time.perf_counter()
                energies.append(d.sweep(m, cutoff=1e-10, krylovdim=krylovdim, maxiter=maxiter))
                ctx.synchronize()
                secs.append(time.perf_counter() - t0)
            prof = {k: ctx.profile(k) for k in kinds}
            ctx.set_profiling(False)
            out[prec] = {"energy": energies[-1], "sweep_energies": energies, "sweep_seconds": secs,
                         "max_bond": max(sum(b.dims) for b in d.bonds), "truncerr": d.truncerr,
                         "kernel_ms": {k: v["ms"] for k, v in prof.items()},
                         "kernel_launches": {k: v["launches"] for k, v in prof.items()}}
        e64, e32 = out["f64"]["energy"], out["tf32x3"]["energy"]
        return {"schedule": {"maxdim": sched, "cutoff": 1e-10, "krylovdim": krylovdim, "maxiter": maxiter},
                "forms": out, "rel_diff_tf32x3_vs_f64": abs(e32 - e64) / abs(e64)}

    # the configuration as specified (5 sweeps: not converged, so the two
    # forms' truncations take different paths), then sweeps to convergence
    spec = run([64, 128, 256, 512, 512], 3, 1)
    conv = run([64, 128, 256, 512] + [512] * 8, 6, 2)
    if rank == 0:
        print(json.dumps({"leg": "dmrg", "model": f"Heisenberg chain N={args.dmrg_n}, OBC, U(1) 2Sz=0, Neel start",
                          "as_specified": spec, "converged": conv}), flush=True)


def j1j2_leg(local: int, maxdim: int = 2048, budget_s: float = 150.0, split: str = "gram", emit=None):
    """Two-site DMRG of the J1-J2 Heisenberg model (J1 = 1, J2 = 0.5) on the
    6 x 6 cylinder (open along x, periodic along y), snake order, N = 36, U(1)
    2Sz = 0, from the Neel state along the snake; the MPO is the automaton
    construction of ``j1j2.J1J2Cylinder``.  Sweeps with maxdim doubling from 64
    to ``maxdim`` (then one more at the maximum), cutoff 1e-10, krylovdim 3,
    maxiter 1, in plain FP64 and in the 3xTF32 form (the H_eff applies on the
    tensor cores, FP64 Rayleigh-quotient energies).  No new FP64 sweep starts
    after ``budget_s`` seconds (the schedule is cut there, and the 3xTF32 form
    runs the same sweeps).  Returns the energies, their relative difference,
    per-sweep seconds and the device time per kernel kind; ``emit(form)`` is
    called with each form's record as soon as it ends."""
    import torch
    import sparsebackends_b200 as sb
    from sparsebackends_b200 import dmrg, j1j2
    torch.cuda.set_device(local)
    kinds = ("gemm", "gemm_thin", "gemm_tc", "tc_pack", "permute", "outer", "axpy", "vector", "other")
    m = j1j2.J1J2Cylinder(6, 6, 1.0, 0.5)
    sched = []
    x = 64
    while x < maxdim:
        sched.append(x)
        x *= 2
    sched += [maxdim] * 2
    out = {}
    for prec in ("f64", "tf32x3"):
        ctx = sb.Context(local)
        d = dmrg.DMRG(m.n, ctx=ctx, precision=prec, device_split=True, mpo=m, split_method=split)
        ctx.set_profiling(True)
        energies, secs = [], []
        t_start = time.perf_counter()
        for mx in sched:
            if prec == "f64" and time.perf_counter() - t_start > budget_s:
                sched = sched[:len(energies)]
                break
            t0 = time.perf_counter()
            energies.append(d.sweep(mx, cutoff=1e-10, krylovdim=3, maxiter=1))
            ctx.synchronize()
            secs.append(time.perf_counter() - t0)
        prof = {k: ctx.profile(k) for k in kinds}
        ctx.set_profiling(False)
        out[prec] = {"energy": energies[-1], "energy_per_site": energies[-1] / m.n, "sweep_energies": energies,
                     "sweep_seconds": secs, "max_bond": max(sum(b.dims) for b in d.bonds), "truncerr": d.truncerr,
                     "kernel_ms": {k: v["ms"] for k, v in prof.items() if v["launches"]},
                     "tc_gemm_tflops_algorithmic": prof["gemm_tc"]["flops"] / (prof["gemm_tc"]["ms"] * 1e-3) / 1e12
                     if prof["gemm_tc"]["ms"] > 0 else None}
        if emit is not None:
            emit({"precision": prec, "maxdim": sched, **out[prec]})
    e64, e32 = out["f64"]["energy"], out["tf32x3"]["energy"]
    return {"model": "J1-J2 Heisenberg (J1=1, J2=0.5), 6x6 cylinder (open x, periodic y), snake order, N=36, "
                     "U(1) 2Sz=0, Neel start",
            "mpo_link": {"charges": m.link.charges, "dims": m.link.dims},
            "schedule": {"maxdim": sched, "cutoff": 1e-10, "krylovdim": 3, "maxiter": 1},
            "split": split, "forms": out, "rel_diff_tf32x3_vs_f64": abs(e32 - e64) / abs(e64)}


def run_j1j2_leg(args, world, rank, local):
    """``j1j2_leg`` with the command line's maxdim, budget and split; each form
    is printed when it ends (a long run cut short keeps what finished)."""
    def emit(form):
        if rank == 0:
            print(json.dumps({"leg": "j1j2_form", **form}), flush=True)
    res = j1j2_leg(local, args.j1j2_maxdim, args.j1j2_budget_s, args.j1j2_split, emit)
    if rank == 0:
        print(json.dumps({"leg": "j1j2", **res}), flush=True)


def run_cpu_leg(args):
    """The CPU restatement of the reference (oracle port: numpy + OpenBLAS) on
    this host's cores, 1 thread and all threads: one chi=2048 matvec (the
    headline workload, uniform zero-padded blocks as the reference stores
    them) and repeated N=16 chi=64 centre-bond matvecs."""
    from threadpoolctl import threadpool_limits
    import sparsebackends_b200 as sb
    from sparsebackends_b200 import dmrg, qn
    layout = workload(args.chi)
    host = host_tensors(layout, args.seed)
    ctx = sb.Context(0)
    lay1, psi1, L1, W1_, R1 = dmrg.canonical_center_problem(ctx)
    host1 = {}
    for name, t in (("psi", psi1), ("L", L1), ("W1", W1_), ("W2", W1_), ("R", R1)):
        u = sb.to_uniform(t)
        host1[name] = (u.keys, np.array(u.data, copy=True))
    out = {"host_cores": os.cpu_count()}
    for threads in (1, blas_threads()):
        row = {}
        for impl, fn in (("cpp", cpp_matvec_rate), ("numpy", cpu_matvec_rate)):
            with threadpool_limits(limits=threads, user_api="blas"):
                r, n, el = fn(layout, host, 0.0, 1)
                r1, n1, el1 = fn(lay1, host1, 5.0, 4000)
            row[impl] = {
                "chi2048": {"value": r, "unit": UNIT, "sample": f"{n} matvec in {el:.1f} s",
                            "gflops_algorithmic": qn.chain_flops(layout, padded=False) * r / 1e9},
                "centre_n16_chi64": {"value": r1, "unit": UNIT, "sample": f"{n1} matvecs in {el1:.1f} s",
                                     "gflops_algorithmic": qn.chain_flops(lay1, padded=False) * r1 / 1e9}}
        out[f"threads_{threads}"] = row
    print(json.dumps({"leg": "cpu", "kind": "port",
                      "what": "restatements of the reference, not the reference itself: cpp = C++ contract_shared! "
                              "(g++ -O3, one OpenBLAS dgemm per block pair), numpy = the oracle (numpy + OpenBLAS)",
                      **out}), flush=True)


def main():
    args = parse()
    world, rank, local = dist_setup(args)
    try:
        if args.impl == "ours" and args.leg == "mixed":
            run_mixed_only(args, world, rank, local)
        elif args.impl == "ours" and args.leg == "dmrg":
            run_dmrg_leg(args, world, rank, local)
        elif args.impl == "ours" and args.leg == "j1j2":
            run_j1j2_leg(args, world, rank, local)
        elif args.impl == "ours" and args.leg == "pxp":
            if rank == 0:
                print(json.dumps({"leg": "pxp", **pxp_leg(local, args.steps, 10.0)}), flush=True)
        elif args.impl == "ours" and args.leg == "cpu":
            if rank == 0:
                run_cpu_leg(args)
        elif args.impl == "reference":
            run_reference(args, world, rank)
        else:
            run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
