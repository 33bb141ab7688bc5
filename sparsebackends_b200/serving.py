"""Serving loop for independent ground-state solves on one GPU.

A request is one two-site DMRG solve of an XXZ chain (``dmrg.DMRG``: N sites,
anisotropy Delta, bond dimension up to chi_max, a fixed number of sweeps).
Requests arrive as a stream (``poisson_arrivals``).  The server keeps several
in flight:

* **slots**: each slot owns a library context, hence its own CUDA stream and
  plan cache, and runs its host work (planning, Lanczos bookkeeping) in a
  thread; library calls release the interpreter lock, so the kernels of the
  requests in flight overlap on the device;
* **admission by memory footprint**: a queued request is started when a slot is
  free and its estimated device footprint (``footprint_bytes``) fits under the
  budget next to the requests in flight, oldest first; a request that alone
  exceeds the budget is rejected before the stream starts;
* **continuous**: a request that arrives while others run is admitted as soon
  as a slot and memory free up, not at batch boundaries.

Every solve keeps its MPS, environments and intermediates on the device for its
whole life.  The kernels are deterministic and a context's plans depend only on
block structure, so a request's result is the same alone and in the mix.
"""
from __future__ import annotations

import math
import threading
import time
from dataclasses import dataclass
from typing import List, Optional

import numpy as np


@dataclass
class Request:
    rid: int
    n: int
    delta: float
    chi_max: int
    sweeps: int = 4
    cutoff: float = 1e-10
    krylovdim: int = 3
    maxiter: int = 1
    arrival: float = 0.0  # seconds after the stream starts


@dataclass
class Result:
    rid: int
    energy: float
    arrival: float
    start: float
    finish: float
    slot: int

    @property
    def latency(self) -> float:
        return self.finish - self.arrival


def footprint_bytes(req: Request) -> int:
    """Upper estimate of a solve's device memory: site tensors (2 chi^2 per
    site), environments (5 chi^2 per bond: the MPO link of the XXZ chain), the
    two-site H_eff intermediates (about 40 chi^2) and Lanczos vectors, in FP64."""
    chi2 = req.chi_max * req.chi_max
    return 8 * chi2 * (2 * req.n + 5 * (req.n + 1) + 40 + 4 * (req.krylovdim + 2))


def poisson_arrivals(requests: List[Request], rate: float, seed: int) -> List[Request]:
    """The same requests with arrival times of a Poisson stream of ``rate``
    requests per second (exponential gaps, seeded)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    t, out = 0.0, []
    for r in requests:
        t += float(rng.exponential(1.0 / rate))
        out.append(Request(**{**r.__dict__, "arrival": t}))
    return out


def random_requests(count: int, seed: int, n_range=(8, 24), chi_range=(8, 64), sweeps: int = 4) -> List[Request]:
    """XXZ chains with Delta ~ U[0.5, 1.5], N ~ U{n_range}, chi_max ~
    log-uniform[chi_range]."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for i in range(count):
        n = int(rng.integers(n_range[0], n_range[1] + 1))
        n += n % 2  # 2Sz = 0 needs an even chain
        delta = float(rng.uniform(0.5, 1.5))
        chi = int(round(math.exp(rng.uniform(math.log(chi_range[0]), math.log(chi_range[1])))))
        out.append(Request(i, n, delta, chi, sweeps))
    return out


def _admit_loop(requests: List[Request], slots: int, budget: int, start_job) -> List[Result]:
    """Replay the stream in real time and admit requests: ``start_job(req, slot,
    on_done)`` starts a solve on a free slot and must call ``on_done(result or
    exception)`` from any thread when it ends."""
    for r in requests:
        if footprint_bytes(r) > budget:
            raise ValueError(f"request {r.rid} needs {footprint_bytes(r)} bytes, over the budget {budget}")
    pending = sorted(requests, key=lambda r: (r.arrival, r.rid))
    free = list(range(slots))
    state = {"used": 0, "running": 0}
    lock = threading.Condition()
    results: List[Result] = []
    errors: List[BaseException] = []

    def done_for(slot: int, fp: int):
        def on_done(res):
            with lock:
                if isinstance(res, BaseException):
                    errors.append(res)
                else:
                    results.append(res)
                free.append(slot)
                state["used"] -= fp
                state["running"] -= 1
                lock.notify_all()
        return on_done

    queued: List[Request] = []
    i = 0
    with lock:
        while i < len(pending) or queued:
            while i < len(pending) and pending[i].arrival <= clock():
                queued.append(pending[i])
                i += 1
            # admit the oldest queued request that fits
            admitted = None
            for q in queued:
                if free and state["used"] + footprint_bytes(q) <= budget:
                    admitted = q
                    break
            if admitted is not None:
                queued.remove(admitted)
                slot, fp = free.pop(0), footprint_bytes(admitted)
                state["used"] += fp
                state["running"] += 1
                start_job(admitted, slot, done_for(slot, fp))
                continue
            # wait for the next arrival or for a request to finish
            timeout: Optional[float] = None
            if i < len(pending):
                timeout = max(0.0, pending[i].arrival - clock())
            lock.wait(timeout=timeout)
        while state["running"] > 0:
            lock.wait()
    if errors:
        raise errors[0]
    return sorted(results, key=lambda r: r.rid)


def clock() -> float:
    """Seconds on the stream clock: time.perf_counter (CLOCK_MONOTONIC on Linux,
    the same clock in every process)."""
    return time.perf_counter()


def _solve(ctx, req: Request, precision: str) -> float:
    from . import dmrg
    d = dmrg.DMRG(req.n, req.delta, ctx, precision=precision)
    e, _ = d.run([req.chi_max] * req.sweeps, cutoff=req.cutoff, krylovdim=req.krylovdim, maxiter=req.maxiter)
    ctx.synchronize()
    return e


def _rebase(requests: List[Request]) -> List[Request]:
    """Arrival times relative to now on the stream clock."""
    t = clock()
    return [Request(**{**r.__dict__, "arrival": r.arrival + t}) for r in requests]


def _relative(results: List[Result], t: float) -> List[Result]:
    return [Result(r.rid, r.energy, r.arrival - t, r.start - t, r.finish - t, r.slot) for r in results]


class Server:
    """``slots`` solves in flight under ``budget_bytes`` of estimated device
    memory, each in ``precision`` ("f64" or "tf32x3"), one thread and one
    library context (stream) per slot."""

    def __init__(self, slots: int = 4, budget_bytes: int = 64 << 30, precision: str = "f64", device: int = 0):
        import sparsebackends_b200 as sb
        self.slots = slots
        self.budget = budget_bytes
        self.precision = precision
        self.ctxs = [sb.Context(device) for _ in range(slots)]

    def solve(self, req: Request, slot: int) -> float:
        return _solve(self.ctxs[slot], req, self.precision)

    def run(self, requests: List[Request]) -> List[Result]:
        """Serve the stream (arrivals in seconds from now); times of the
        returned Results are relative to the stream's start."""
        t = clock()
        stream = _rebase(requests)

        def start_job(req, slot, on_done):
            t_start = clock()

            def work():
                try:
                    e = self.solve(req, slot)
                    on_done(Result(req.rid, e, req.arrival, t_start, clock(), slot))
                except BaseException as exc:  # reported after the stream
                    on_done(exc)
            threading.Thread(target=work, daemon=True).start()

        return _relative(_admit_loop(stream, self.slots, self.budget, start_job), t)


def summary(results: List[Result]) -> dict:
    """solves/s over the span from the first arrival to the last finish, and
    nearest-rank p50 / p99 latency (arrival to finish, queueing included)."""
    lat = sorted(r.latency for r in results)
    span = max(r.finish for r in results) - min(r.arrival for r in results)

    def pct(p):
        return lat[max(0, math.ceil(p / 100.0 * len(lat)) - 1)]

    return {"requests": len(results), "solves_per_s": len(results) / span, "p50_ms": 1e3 * pct(50),
            "p99_ms": 1e3 * pct(99), "span_s": span}
