"""Host logic of the serving loop (no GPU): arrivals, footprints, admission
order and the latency summary, with the solve replaced by a stub."""
import threading
import time

from sparsebackends_b200 import serving


class StubServer(serving.Server):
    def __init__(self, slots, budget):
        self.slots, self.budget, self.precision = slots, budget, "f64"
        self.ctxs = [None] * slots
        self.active, self.peak, self.peak_mem, self.mem = 0, 0, 0, 0
        self.lock = threading.Lock()

    def solve(self, req, slot):
        fp = serving.footprint_bytes(req)
        with self.lock:
            self.active += 1
            self.mem += fp
            self.peak = max(self.peak, self.active)
            self.peak_mem = max(self.peak_mem, self.mem)
        time.sleep(0.02 + 0.001 * req.n)
        with self.lock:
            self.active -= 1
            self.mem -= fp
        return -0.4 * req.n


def test_poisson_arrivals_are_seeded_and_increasing():
    reqs = serving.random_requests(20, seed=3)
    a = serving.poisson_arrivals(reqs, rate=50.0, seed=1)
    b = serving.poisson_arrivals(reqs, rate=50.0, seed=1)
    assert [r.arrival for r in a] == [r.arrival for r in b]
    assert all(x.arrival < y.arrival for x, y in zip(a, a[1:]))
    assert all(r.n % 2 == 0 and 8 <= r.n <= 24 and 8 <= r.chi_max <= 64 for r in reqs)


def test_admission_respects_slots_and_memory_budget():
    reqs = serving.poisson_arrivals(serving.random_requests(24, seed=5), rate=200.0, seed=2)
    budget = 3 * max(serving.footprint_bytes(r) for r in reqs)
    srv = StubServer(slots=4, budget=budget)
    res = srv.run(reqs)
    assert [r.rid for r in res] == list(range(24))
    assert srv.peak <= 4 and srv.peak_mem <= budget
    assert srv.peak >= 2  # requests overlap
    assert all(r.start >= r.arrival - 1e-9 and r.finish >= r.start for r in res)
    s = serving.summary(res)
    assert s["requests"] == 24 and s["p50_ms"] <= s["p99_ms"]


def test_oversized_request_is_rejected():
    reqs = serving.random_requests(2, seed=7)
    srv = StubServer(slots=2, budget=serving.footprint_bytes(reqs[0]) - 1)
    try:
        srv.run(reqs)
    except ValueError:
        return
    raise AssertionError("expected a ValueError")
