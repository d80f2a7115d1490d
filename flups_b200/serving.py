"""Serving loop for many Poisson solves of different sizes and boundary
conditions on one GPU.

Requests (grid size, boundary conditions, Green's kernel, precision, a
right-hand side already in device memory) arrive over time.  The server keeps
set-up solvers -- plans and the Green's spectrum resident in HBM -- in a cache
keyed by (grid, BCs, kernel, precision), so only the first request of a key
pays the set-up.  It admits work by HBM footprint: a key's solver, its work
arrays for the batch and the batch's staging arrays must fit in the memory
budget.  A batch shrinks (halving) until it fits in what is free; only when
not even a single solve fits are idle solvers evicted, least-recently-used
first, so a burst does not trade resident solvers (and their set-up time)
for larger batches.  Continuous batching: every key has at most one batch in flight on its
own CUDA stream; requests that arrive meanwhile queue and go out together
(one flups_solve_batch launch per pass) as soon as the key's previous batch
completes, while other keys' batches run concurrently on their streams.
Latency is measured from a request's arrival to the completion of its batch.

The device side is a backend object so that the scheduling logic (admission,
eviction, batching) runs on the CPU under test with a fake backend.
"""
import collections
import time

import numpy as np


class Request:
    __slots__ = ("rid", "key", "rhs", "out", "t_arrival", "t_done", "batch")

    def __init__(self, rid, key, rhs, out, t_arrival):
        self.rid, self.key, self.rhs, self.out = rid, key, rhs, out
        self.t_arrival, self.t_done, self.batch = t_arrival, None, 0


class Server:
    """Scheduling loop over a backend.

    backend.make(key) -> handle        set-up solver (may take time)
    backend.footprint(key, nbatch)     device bytes a handle needs for nbatch
    backend.launch(handle, reqs)       queue one batched solve, asynchronous
    backend.done(handle) -> bool       the handle's last launch completed
    backend.finish(handle, reqs)       results of the completed launch are in place
    backend.free(handle)               release the handle's device memory
    """

    def __init__(self, backend, budget_bytes, max_batch=16, max_inflight=None, clock=time.perf_counter):
        self.b = backend
        self.budget = int(budget_bytes)
        self.max_batch = int(max_batch)
        self.max_inflight = max_inflight   # None: one batch per key at a time, keys concurrent
        self.clock = clock
        self.cache = collections.OrderedDict()   # key -> handle (LRU order)
        self.reserved = {}                         # key -> bytes held
        self.inflight = {}                         # key -> list of requests
        self.queues = collections.defaultdict(collections.deque)
        self.completed = []
        self.setups = 0
        self.evictions = 0
        self.batches = 0

    # ---------------------------------------------------------------- memory
    def used(self):
        return sum(self.reserved.values())

    def _evict_for(self, need):
        """Evict idle cached keys (LRU first) until `need` more bytes fit."""
        for key in list(self.cache.keys()):
            if self.used() + need <= self.budget:
                break
            if key in self.inflight:
                continue
            self.b.free(self.cache.pop(key))
            self.reserved.pop(key, None)
            self.evictions += 1
        return self.used() + need <= self.budget

    def _admit(self, key, nbatch):
        """(handle, nb) for key with the largest batch nb <= nbatch that fits
        without evicting another key, or after evicting idle keys for a single
        solve when nothing fits; (None, 0) while memory is short."""
        have = self.reserved.get(key, 0)
        free = self.budget - self.used()
        nb = nbatch
        while nb >= 1:
            need = self.b.footprint(key, nb)
            if need - have <= free:
                break
            nb = nb // 2 if nb > 1 else 0
        if nb == 0:
            nb = 1
            need = self.b.footprint(key, 1)
            if not self._evict_for(need - have):
                return None, 0
        if key not in self.cache:
            self.cache[key] = self.b.make(key)
            self.setups += 1
        self.cache.move_to_end(key)
        self.reserved[key] = max(have, need)
        return self.cache[key], nb

    # ---------------------------------------------------------------- loop
    def submit(self, req):
        self.queues[req.key].append(req)

    def poll(self):
        """Retire completed batches, then launch a batch for every idle key with
        waiting requests that fits in memory.  Returns the number launched."""
        now = None
        for key in list(self.inflight):
            h = self.cache[key]
            if self.b.done(h):
                reqs = self.inflight.pop(key)
                self.b.finish(h, reqs)
                now = self.clock() if now is None else now
                for r in reqs:
                    r.t_done = now
                self.completed.extend(reqs)
        launched = 0
        # oldest waiting request first
        order = sorted((q[0].t_arrival, k) for k, q in self.queues.items() if q and k not in self.inflight)
        for _, key in order:
            if self.max_inflight is not None and len(self.inflight) >= self.max_inflight:
                break
            q = self.queues[key]
            h, nb = self._admit(key, min(len(q), self.max_batch))
            if h is None:
                continue
            reqs = [q.popleft() for _ in range(nb)]
            for r in reqs:
                r.batch = nb
            self.b.launch(h, reqs)
            self.inflight[key] = reqs
            self.batches += 1
            launched += 1
        return launched

    def idle(self):
        return not self.inflight and not any(self.queues.values())

    def close(self):
        for h in self.cache.values():
            self.b.free(h)
        self.cache.clear()
        self.reserved.clear()


def run_trace(server, trace, make_request, spin=None):
    """Feed `trace` (list of (t_arrival_s, key, payload)) in real time.
    make_request(i, key, payload, t_arrival) -> Request.  Returns wall seconds."""
    t0 = server.clock()
    i, n = 0, len(trace)
    while i < n or not server.idle():
        now = server.clock() - t0
        while i < n and trace[i][0] <= now:
            ta, key, payload = trace[i]
            server.submit(make_request(i, key, payload, t0 + ta))
            i += 1
        if server.poll() == 0 and spin is not None:
            spin()
    return server.clock() - t0


def latency_stats(reqs):
    lat = np.array([r.t_done - r.t_arrival for r in reqs]) * 1e3
    return {"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_ms": float(lat.mean()), "max_ms": float(lat.max())}


# ---------------------------------------------------------------- the GPU backend
BC_SETS = {
    "UNB3": [["UNB", "UNB"]] * 3,
    "PER2_UNB": [["PER", "PER"], ["PER", "PER"], ["UNB", "UNB"]],
    "EVEN_UNB2": [["EVEN", "EVEN"], ["UNB", "UNB"], ["UNB", "UNB"]],
}


class GpuBackend:
    """Set-up solvers (pyflups) with their own CUDA stream each; batches are
    gathered into a per-key input array, solved with flups_solve_batch in
    async mode, and scattered back to the requests' output arrays on the same
    stream; completion is a CUDA event."""

    def __init__(self, device=0, autotune=False):
        import torch
        from flups_b200 import pyflups as pf
        self.torch, self.pf = torch, pf
        self.dev = torch.device("cuda", device)
        self.autotune = autotune

    def make(self, key):
        n, bcs, kernel, prec = key
        pf, torch = self.pf, self.torch
        B = pf.BoundaryType
        t = pf.Topology(0, 1, [n, n, n])
        s = pf.Solver(t, [[B[a], B[b]] for a, b in BC_SETS[bcs]], [1.0 / n] * 3, [1.0] * 3)
        s.set_green_type(pf.GreenType[kernel])
        s.set_precision(prec)
        st = torch.cuda.Stream(device=self.dev)
        s.set_stream(st)
        s.set_async(True)
        s.set_autotune(self.autotune)
        s.setup()
        return {"key": key, "topo": t, "solver": s, "stream": st, "event": None, "bin": None, "bout": None}

    def footprint(self, key, nbatch):
        """Work arrays for nbatch, the Green's spectrum and twiddles (the all-UNB
        sizes, padded rows included, bound the other BC sets from above), plus
        the gather / scatter arrays of a batch."""
        n, _, _, prec = key
        w = 4 if prec == 32 else 8
        pitch = -(-(n + 1) // (128 // (2 * w))) * (128 // (2 * w))   # padded complex row
        work = 2 * w * pitch * n * n * 3 * nbatch                      # states 1 and 2
        green = w * (-(-(n + 1) // 32) * 32) * (n + 1) * (n + 1)
        batch = 2 * 8 * n ** 3 * nbatch if nbatch > 1 else 0
        return work + green + batch + (1 << 20)

    def launch(self, h, reqs):
        torch = self.torch
        s, st = h["solver"], h["stream"]
        nb = len(reqs)
        with torch.cuda.stream(st):
            if nb == 1:
                s.solve(reqs[0].out, reqs[0].rhs)
            else:
                n = h["key"][0]
                if h["bin"] is None or h["bin"].shape[0] < nb:
                    h["bin"] = torch.empty((nb, n, n, n), dtype=torch.float64, device=self.dev)
                    h["bout"] = torch.empty_like(h["bin"])
                bin_, bout = h["bin"][:nb], h["bout"][:nb]
                for k, r in enumerate(reqs):
                    bin_[k].copy_(r.rhs)
                s.solve_batch(bout, bin_, nb)
                for k, r in enumerate(reqs):
                    r.out.copy_(bout[k])
            ev = torch.cuda.Event()
            ev.record(st)
        h["event"] = ev

    def done(self, h):
        return h["event"] is None or h["event"].query()

    def finish(self, h, reqs):
        pass

    def free(self, h):
        h["event"] = None
        h["solver"] = None
        h["topo"] = None
        h["bin"] = h["bout"] = None


def rhs_pool(sizes, per_size=4, device=None, seed=2):
    """Seeded sums of 8 Gaussians (centres uniform in the domain shrunk by 0.2
    per side, sigma uniform in [0.03, 0.08], amplitude uniform in [-1, 1]) on
    the device, per_size per grid size: {(n, idx): tensor [z][y][x]}."""
    import torch
    pool = {}
    for n in sizes:
        xs = torch.tensor((np.arange(n) + 0.5) / n, dtype=torch.float64, device=device)
        for idx in range(per_size):
            rng = np.random.default_rng([seed, n, idx])
            f = torch.zeros((n, n, n), dtype=torch.float64, device=device)
            for _ in range(8):
                c = rng.uniform(0.2, 0.8, 3)
                sg = rng.uniform(0.03, 0.08)
                a = rng.uniform(-1.0, 1.0)
                gx = torch.exp(-(xs - c[0]) ** 2 / sg ** 2)
                gy = torch.exp(-(xs - c[1]) ** 2 / sg ** 2)
                gz = torch.exp(-(xs - c[2]) ** 2 / sg ** 2)
                f += a * gz[:, None, None] * gy[None, :, None] * gx[None, None, :]
            pool[(n, idx)] = f
    return pool


def make_trace(n_req=2000, rate=500.0, seed=5, sizes=(32, 48, 64, 96, 128, 192, 256)):
    """Poisson arrivals at `rate`/s; size, BC set, kernel uniform; precision 32/64 at 0.8/0.2."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, n_req))
    trace = []
    for i in range(n_req):
        n = int(rng.choice(sizes))
        bcs = str(rng.choice(list(BC_SETS)))
        kernel = str(rng.choice(["HEJ_2", "LGF_2"]))
        prec = 32 if rng.random() < 0.8 else 64
        trace.append((float(t[i]), (n, bcs, kernel, prec), int(rng.integers(0, 4))))
    return trace
