"""Exchange steps of the z-slab decomposed solve (flups_b200/slab.py) across
processes on CPU: gloo, world_size 2 and 3, with spectra whose values encode
(plane, row, column, part), so every moved block is checked in place: the
forward exchange from plane arrays into column arrays, the backward one
from column arrays into plane arrays."""
import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent
SHAPE = (10, 6, 16, 2)   # planes, rows, padded columns, (re, im)
NX = 13                  # spectrum columns in use


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _code(torch):
    z, y, x, c = torch.meshgrid(*[torch.arange(n, dtype=torch.float64) for n in SHAPE], indexing="ij")
    return 1 + z * 1e6 + y * 1e4 + x * 10 + c


def _worker(rank, world, port, q):
    sys.path.insert(0, str(ROOT))
    import datetime

    import torch
    import torch.distributed as dist

    from flups_b200.slab import (ProcessGroupTransport, SlabPlan, pack_backward, pack_forward, recv_shapes_backward,
                                 recv_shapes_forward, unpack_backward, unpack_forward)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        plan = SlabPlan(SHAPE[0], NX, world)
        t = ProcessGroupTransport()
        code = _code(torch)
        z0, z1 = plan.z[rank]
        x0, x1 = plan.x[rank]
        cp = (x1 - x0 + 3) // 4 * 4
        # after the forward passes a rank's plane array holds its planes
        planes = code[z0:z1].clone()
        columns = torch.full((SHAPE[0], SHAPE[1], cp, SHAPE[3]), -1.0, dtype=torch.float64)
        recv = t.alltoall(pack_forward(planes, plan, rank), recv_shapes_forward(columns, plan, rank))
        unpack_forward(columns, plan, rank, recv)
        ok_fwd = bool(torch.equal(columns[:, :, :x1 - x0], code[:, :, x0:x1]))
        # the last-direction pass changes this rank's columns over every plane
        columns[:, :, :x1 - x0] = -code[:, :, x0:x1]
        planes.fill_(0.0)
        recv = t.alltoall(pack_backward(columns, plan, rank), recv_shapes_backward(planes, plan, rank))
        unpack_backward(planes, plan, rank, recv)
        ok_bwd = bool(torch.equal(planes[:, :, :NX], -code[z0:z1, :, :NX]))
        # the same exchanges through reusable flat send / receive buffers
        sbuf = torch.empty(4096, dtype=torch.float64)
        rbuf = torch.empty(4096, dtype=torch.float64)
        planes = code[z0:z1].clone()
        columns.fill_(-1.0)
        recv = t.alltoall(pack_forward(planes, plan, rank, sbuf), recv_shapes_forward(columns, plan, rank), sbuf, rbuf)
        unpack_forward(columns, plan, rank, recv)
        ok_fwd = ok_fwd and bool(torch.equal(columns[:, :, :x1 - x0], code[:, :, x0:x1]))
        columns[:, :, :x1 - x0] = -code[:, :, x0:x1]
        planes.fill_(0.0)
        recv = t.alltoall(pack_backward(columns, plan, rank, sbuf), recv_shapes_backward(planes, plan, rank), sbuf, rbuf)
        unpack_backward(planes, plan, rank, recv)
        ok_bwd = ok_bwd and bool(torch.equal(planes[:, :, :NX], -code[z0:z1, :, :NX]))
        q.put((rank, ok_fwd, ok_bwd))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_slab_exchanges_gloo(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[0] for r in res] == list(range(world))
    assert all(r[1] for r in res), "forward exchange: a rank's columns over every plane"
    assert all(r[2] for r in res), "backward exchange: a rank's planes over every column"


def test_slab_plan_covers_everything():
    from flups_b200.slab import SlabPlan
    for nz, nx, w in [(512, 513, 1), (512, 513, 3), (7, 5, 5), (64, 33, 4)]:
        p = SlabPlan(nz, nx, w)
        assert p.z[0][0] == 0 and p.z[-1][1] == nz and p.x[0][0] == 0 and p.x[-1][1] == nx
        assert all(p.z[k][1] == p.z[k + 1][0] and p.x[k][1] == p.x[k + 1][0] for k in range(w - 1))
        assert all(b > a for a, b in p.z + p.x)
    with pytest.raises(ValueError):
        SlabPlan(4, 100, 5)
