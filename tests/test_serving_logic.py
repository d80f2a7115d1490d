"""Scheduling logic of the serving loop (flups_b200/serving.py) on the CPU
with a fake backend: every request completes, requests that arrive while
their key is busy are batched (up to max_batch), keys run concurrently,
admission waits while memory is short, and idle solvers are evicted least
recently used when a new key needs room."""
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))

from flups_b200.serving import Request, Server  # noqa: E402


class FakeBackend:
    def __init__(self, per_key_bytes=100, per_rhs_bytes=10, steps=2):
        self.per_key, self.per_rhs, self.steps = per_key_bytes, per_rhs_bytes, steps
        self.made, self.freed, self.launches = [], [], []

    def make(self, key):
        self.made.append(key)
        return {"key": key, "left": 0}

    def footprint(self, key, nb):
        return self.per_key + self.per_rhs * nb

    def launch(self, h, reqs):
        self.launches.append((h["key"], len(reqs)))
        h["left"] = self.steps

    def done(self, h):
        h["left"] -= 1
        return h["left"] < 0

    def finish(self, h, reqs):
        for r in reqs:
            r.out.append(r.rid)

    def free(self, h):
        self.freed.append(h["key"])


class Clock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        return self.t


def _req(i, key, t):
    return Request(i, key, None, [], t)


def test_batches_and_completes():
    clk = Clock()
    be = FakeBackend()
    srv = Server(be, budget_bytes=10_000, max_batch=4, clock=clk)
    for i in range(10):
        srv.submit(_req(i, "A", 0.0))
    srv.submit(_req(10, "B", 0.0))
    for _ in range(50):
        clk.t += 1
        srv.poll()
    assert srv.idle()
    assert sorted(r.rid for r in srv.completed) == list(range(11))
    assert all(r.out == [r.rid] for r in srv.completed)
    sizes = [nb for k, nb in be.launches if k == "A"]
    assert sizes == [4, 4, 2]
    # B ran while A's batches were in flight
    first_b = next(i for i, (k, _) in enumerate(be.launches) if k == "B")
    assert first_b == 1
    assert be.made.count("A") == 1 and srv.setups == 2


def test_admission_waits_and_evicts_lru():
    clk = Clock()
    be = FakeBackend(per_key_bytes=100, per_rhs_bytes=0, steps=0)
    srv = Server(be, budget_bytes=250, max_batch=1, clock=clk)
    for i, key in enumerate(["A", "B", "C"]):
        srv.submit(_req(i, key, float(i)))
    clk.t = 1
    srv.poll()   # A and B fit, C waits (A, B in flight)
    assert set(srv.inflight) == {"A", "B"}
    assert len(srv.queues["C"]) == 1
    clk.t = 2
    srv.poll()   # A, B done -> idle; C evicts the least recently used (A)
    assert be.freed == ["A"]
    assert "C" in srv.inflight
    for _ in range(3):
        clk.t += 1
        srv.poll()
    assert srv.idle() and len(srv.completed) == 3
    assert srv.used() <= 250


def test_serial_mode_one_at_a_time():
    clk = Clock()
    be = FakeBackend()
    srv = Server(be, budget_bytes=10_000, max_batch=1, max_inflight=1, clock=clk)
    for i in range(5):
        srv.submit(_req(i, "AB"[i % 2], 0.0))
    while not srv.idle():
        clk.t += 1
        srv.poll()
        assert len(srv.inflight) <= 1
    assert all(nb == 1 for _, nb in be.launches)
    assert len(srv.completed) == 5


def test_batch_shrinks_before_evicting():
    """Under a burst a resident key's batch is cut to what fits in the free
    budget instead of evicting another resident solver."""
    clk = Clock()
    be = FakeBackend(per_key_bytes=100, per_rhs_bytes=10, steps=0)
    srv = Server(be, budget_bytes=260, max_batch=8, clock=clk)
    srv.submit(_req(0, "A", 0.0))
    srv.submit(_req(1, "B", 0.0))
    clk.t = 1
    srv.poll()   # A and B resident at one rhs each: 220 bytes
    for _ in range(3):
        clk.t += 1
        srv.poll()
    assert srv.idle() and srv.used() == 220
    for i in range(8):
        srv.submit(_req(2 + i, "A", clk.t))
    while not srv.idle():
        clk.t += 1
        srv.poll()
    # 40 bytes free: A grows to 4 rhs at most (150 of 260 with B's 110)
    sizes = [nb for k, nb in be.launches if k == "A"][1:]
    assert sizes == [4, 4]
    assert be.freed == [] and srv.evictions == 0 and srv.setups == 2
    assert srv.used() <= 260
