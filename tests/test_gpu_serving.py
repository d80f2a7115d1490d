"""Continuous batching on the GPU: a burst of requests of mixed grid sizes,
boundary conditions, kernels and precisions goes through the serving loop
(batched launches, keys overlapping on their streams); every result must be
the same, bit for bit, as the same request solved alone by a fresh solver."""
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))

pytestmark = pytest.mark.gpu


def test_mix_equals_alone():
    import torch
    from flups_b200.serving import GpuBackend, Request, Server, make_trace, rhs_pool, run_trace
    sizes = (32, 48, 64)
    pool = rhs_pool(sizes, per_size=2, device="cuda")
    torch.cuda.synchronize()
    trace = make_trace(n_req=48, rate=20000.0, seed=7, sizes=sizes)
    trace = [(t, key, idx % 2) for t, key, idx in trace]
    be = GpuBackend()
    srv = Server(be, budget_bytes=8 << 30, max_batch=8)

    def make(i, key, idx, ta):
        rhs = pool[(key[0], idx)]
        return Request(i, key, rhs, torch.empty_like(rhs), ta)

    run_trace(srv, trace, make)
    torch.cuda.synchronize()
    assert len(srv.completed) == len(trace)
    assert max(r.batch for r in srv.completed) > 1          # batching happened
    alone = {}
    for r in srv.completed:
        h = alone.get(r.key) or be.make(r.key)
        alone[r.key] = h
        out = torch.empty_like(r.rhs)
        with torch.cuda.stream(h["stream"]):
            h["solver"].solve(out, r.rhs)
        h["stream"].synchronize()
        assert torch.equal(out, r.out), f"request {r.rid} {r.key} differs in the mix"
    srv.close()
