"""A solve split over ranks by planes of the last direction (z).

The reference distributes a solve over MPI ranks as pencils and moves the
data between the directions with all-to-all exchanges (Solver.cpp:629-715,
SwitchTopoX_a2a.cpp:118-247).  Here every array stays x-fastest and the
decomposition needs one transpose each way:

  rank r owns user planes [z0, z1) and spectrum columns [x0, x1);
  1. x and y forward passes of its planes           (flups_b200_slab_forward)
  2. all-to-all: the block (its planes, columns of rank j) goes to rank j,
     so rank r holds its columns over every plane
  3. last-direction pass (forward DFT, Green's multiply, inverse DFT) of its
     columns                                         (flups_b200_slab_fused)
  4. all-to-all back: the block (planes of rank j, its columns) goes to rank j
  5. y and x inverse passes of its planes           (flups_b200_slab_backward)

Each step is the single-GPU pass restricted to a slab, so the result equals
the one-rank solve bit for bit.  A rank's solver holds its planes (the plane
array), its columns over every plane (the column array) and its columns of
the Green's spectrum, so its device memory falls with the rank count.  The user arrays of a rank hold its planes only.  Scalar fields
(lda 1), STD solves, x, y and z transformed in that order.

The exchanges take any transport with `alltoall(sends, recv_shapes)`:
ProcessGroupTransport (torch.distributed: NCCL between GPUs, gloo on CPU),
or the in-process exchange of `solve_local` (several ranks' solvers on one
device).
"""


def split(n, parts, k):
    """Balanced range [lo, hi) of part k of n items."""
    return (k * n) // parts, ((k + 1) * n) // parts


class SlabPlan:
    """Planes and spectrum columns of every rank."""

    def __init__(self, nz_user, nx_spec, world):
        if world < 1 or world > nz_user or world > nx_spec:
            raise ValueError(f"{world} ranks for {nz_user} planes and {nx_spec} spectrum columns")
        self.world = world
        self.z = [split(nz_user, world, k) for k in range(world)]
        self.x = [split(nx_spec, world, k) for k in range(world)]


# ---------------------------------------------------------------- exchanges
# planes: this rank's plane array (nz_r, ny, pitch, 2) (complex values as
# pairs), columns: its column array (nz, ny, cpitch, 2); spectrum columns
# x < nx_spec are in use.

def _pack(blocks, out):
    """The blocks as new contiguous tensors, or copied into consecutive
    segments of the flat tensor `out` (one copy, no concatenation after)."""
    if out is None:
        return [b.contiguous() for b in blocks]
    views, off = [], 0
    for b in blocks:
        v = out[off:off + b.numel()].view(b.shape)
        v.copy_(b)
        views.append(v)
        off += b.numel()
    return views


def pack_forward(planes, plan, rank, out=None):
    """Blocks (this rank's planes, columns of rank j) for every j."""
    return _pack([planes[:, :, a:b] for a, b in plan.x], out)


def unpack_forward(columns, plan, rank, recvs):
    """recvs[i]: block (planes of rank i, this rank's columns) from rank i."""
    a, b = plan.x[rank]
    for i, (z0, z1) in enumerate(plan.z):
        columns[z0:z1, :, :b - a].copy_(recvs[i].view(z1 - z0, columns.shape[1], b - a, columns.shape[3]))


def pack_backward(columns, plan, rank, out=None):
    """Blocks (planes of rank j, this rank's columns) for every j."""
    a, b = plan.x[rank]
    return _pack([columns[z0:z1, :, :b - a] for z0, z1 in plan.z], out)


def unpack_backward(planes, plan, rank, recvs):
    """recvs[j]: block (this rank's planes, columns of rank j) from rank j."""
    z0, z1 = plan.z[rank]
    for j, (a, b) in enumerate(plan.x):
        planes[:, :, a:b].copy_(recvs[j].view(z1 - z0, planes.shape[1], b - a, planes.shape[3]))


def recv_shapes_forward(columns, plan, rank):
    a, b = plan.x[rank]
    return [(z1 - z0, columns.shape[1], b - a, columns.shape[3]) for z0, z1 in plan.z]


def recv_shapes_backward(planes, plan, rank):
    z0, z1 = plan.z[rank]
    return [(z1 - z0, planes.shape[1], b - a, planes.shape[3]) for a, b in plan.x]


class ProcessGroupTransport:
    """all-to-all through torch.distributed (one flat all_to_all_single)."""

    def __init__(self, group=None):
        import torch
        import torch.distributed as dist
        self.torch, self.dist, self.group = torch, dist, group

    def alltoall(self, sends, recv_shapes, send_flat=None, recv_flat=None):
        """sends: the blocks for every rank (consecutive views of `send_flat`
        when it is given, else concatenated here); returns the received
        blocks (views of `recv_flat` when it is given)."""
        torch = self.torch
        send = send_flat if send_flat is not None else torch.cat([s.reshape(-1) for s in sends])
        sizes_in = [s.numel() for s in sends]
        sizes_out = [a * b * c * d for a, b, c, d in recv_shapes]
        recv = recv_flat[:sum(sizes_out)] if recv_flat is not None else \
            torch.empty(sum(sizes_out), dtype=send.dtype, device=send.device)
        self.dist.all_to_all_single(recv, send[:sum(sizes_in)], sizes_out, sizes_in, group=self.group)
        return list(torch.split(recv, sizes_out))


# ---------------------------------------------------------------- one rank

class SlabRank:
    """One rank's share of a z-slab decomposed solve: takes a pyflups Solver
    that is initialised (green type, precision set) but not set up, gives it
    its planes and columns and sets it up."""

    def __init__(self, solver, rank, world):
        import torch
        self.torch = torch
        self.s, self.rank, self.world = solver, rank, world
        code, (nx, ny, nz), pitch, nz_user, _, es = solver.slab_info()
        if code != 0:
            raise ValueError("this solver cannot run a z-slab solve (3-D, scalar, STD, directions x, y, z in order)")
        self.plan = SlabPlan(nz_user, nx, world)
        self.z0, self.z1 = self.plan.z[rank]
        self.x0, self.x1 = self.plan.x[rank]
        self._ok(solver.slab_own(self.z0, self.z1, self.x0, self.x1), "slab_own")
        solver.setup()
        code, _, _, _, cpitch, _ = solver.slab_info()
        self.dtype = torch.float32 if es == 4 else torch.float64
        self.planes_shape = (self.z1 - self.z0, ny, pitch, 2)
        self.columns_shape = (nz, ny, cpitch, 2)

    def _view(self, ptr, shape):
        torch = self.torch
        if not ptr:
            raise RuntimeError("no work array (set up?)")
        iface = {"shape": shape, "typestr": "<f4" if self.dtype == torch.float32 else "<f8",
                 "data": (ptr, False), "version": 3}

        class _View:
            __cuda_array_interface__ = iface

        return torch.as_tensor(_View(), device="cuda")

    def planes(self):
        """The plane array (owned planes of the spectrum between the passes) as a device tensor."""
        return self._view(self.s.slab_planes_ptr(), self.planes_shape)

    def columns(self):
        """The column array (owned columns over every plane) as a device tensor."""
        return self._view(self.s.slab_columns_ptr(), self.columns_shape)

    def _ok(self, code, what):
        if code != 0:
            raise RuntimeError(f"{what} failed with code {code} (last CUDA error {self.s.last_error()})")

    def forward(self, rhs):
        """rhs: this rank's planes of the right-hand side (device array, user layout)."""
        self._ok(self.s.slab_forward(rhs), "slab forward")
        self.s.synchronize()

    def fused(self):
        self._ok(self.s.slab_fused(), "slab last-direction pass")
        self.s.synchronize()

    def backward(self, field):
        """field: this rank's planes of the result (device array, user layout)."""
        self._ok(self.s.slab_backward(field), "slab backward")
        self.s.synchronize()

    def solve(self, field, rhs, transport):
        """The whole solve of this rank; every rank calls it with the same transport group."""
        torch = self.torch
        planes, columns = self.planes(), self.columns()
        if getattr(self, "_flat", None) is None:
            # exchange buffers, kept: the largest block set a rank sends or receives
            nx = self.plan.x[-1][1]
            ny = self.planes_shape[1]
            own = (self.z1 - self.z0) * ny * nx * 2
            cols = self.columns_shape[0] * ny * (self.x1 - self.x0) * 2
            self._flat = (torch.empty(max(own, cols), dtype=self.dtype, device=planes.device),
                          torch.empty(max(own, cols), dtype=self.dtype, device=planes.device))
        sbuf, rbuf = self._flat
        self.forward(rhs)
        recv = transport.alltoall(pack_forward(planes, self.plan, self.rank, sbuf),
                                  recv_shapes_forward(columns, self.plan, self.rank), sbuf, rbuf)
        unpack_forward(columns, self.plan, self.rank, recv)
        torch.cuda.synchronize()
        self.fused()
        recv = transport.alltoall(pack_backward(columns, self.plan, self.rank, sbuf),
                                  recv_shapes_backward(planes, self.plan, self.rank), sbuf, rbuf)
        unpack_backward(planes, self.plan, self.rank, recv)
        torch.cuda.synchronize()
        self.backward(field)


def _split_table(plan):
    """Column split of the ranks: xs[j] = first column of rank j, xs[world] = columns."""
    return [a for a, _ in plan.x] + [plan.x[-1][1]]


def connect_local(ranks):
    """Several ranks' solvers in one process (one device): every rank's y
    passes use the column arrays of all of them directly."""
    cols = [r.s.slab_columns_ptr() for r in ranks]
    pitches = [r.columns_shape[2] for r in ranks]
    for r in ranks:
        r._ok(r.s.slab_peers(cols, _split_table(r.plan), pitches), "slab_peers")


def connect_peers(rank, group=None):
    """One rank per GPU: open every other rank's column array through CUDA
    IPC (peer memory over NVLink) so this rank's y passes store into and
    load from them directly.  Collective over the group."""
    import ctypes

    import torch.distributed as dist
    from flups_b200 import pyflups as pf
    lib = pf.load_library()
    mine = rank.s.slab_columns_ptr()
    h = ctypes.create_string_buffer(64)
    rank._ok(lib.flups_b200_ipc_handle(ctypes.c_void_p(mine), h), "ipc handle")
    entries = [None] * rank.world
    dist.all_gather_object(entries, (rank.rank, bytes(h.raw), rank.columns_shape[2]), group=group)
    cols, pitches, opened = [], [], []
    for j, hb, pitch in sorted(entries):
        if j == rank.rank:
            cols.append(mine)
        else:
            ptr = ctypes.c_void_p()
            rank._ok(lib.flups_b200_ipc_open(ctypes.create_string_buffer(hb, 64), ctypes.byref(ptr)), "ipc open")
            cols.append(ptr.value)
            opened.append(ptr.value)
        pitches.append(pitch)
    rank._ok(rank.s.slab_peers(cols, _split_table(rank.plan), pitches), "slab_peers")
    rank._opened = opened
    return opened


def solve_connected(rank, field, rhs, group=None):
    """The solve of one rank per GPU after connect_peers: the y passes move
    the spectrum between the GPUs themselves; barriers order the steps."""
    import torch.distributed as dist
    torch = rank.torch
    rank.forward(rhs)
    torch.cuda.synchronize()
    dist.barrier(group=group)
    rank.fused()
    dist.barrier(group=group)
    rank.backward(field)
    torch.cuda.synchronize()
    dist.barrier(group=group)


def solve_local_connected(ranks, fields, rhss):
    """solve_connected for several ranks' solvers in one process (after connect_local)."""
    torch = ranks[0].torch
    for r, rhs in zip(ranks, rhss):
        r.forward(rhs)
    torch.cuda.synchronize()
    for r in ranks:
        r.fused()
    torch.cuda.synchronize()
    for r, f in zip(ranks, fields):
        r.backward(f)
    torch.cuda.synchronize()


def solve_local(ranks, fields, rhss):
    """The decomposed solve of several ranks' solvers in one process (one
    device): the same steps, with the all-to-all done by device copies."""
    torch = ranks[0].torch
    planes = [r.planes() for r in ranks]
    columns = [r.columns() for r in ranks]
    for r, rhs in zip(ranks, rhss):
        r.forward(rhs)
    sends = [pack_forward(p, r.plan, r.rank) for r, p in zip(ranks, planes)]
    for r, c in zip(ranks, columns):
        unpack_forward(c, r.plan, r.rank, [sends[i][r.rank] for i in range(len(ranks))])
    torch.cuda.synchronize()
    for r in ranks:
        r.fused()
    sends = [pack_backward(c, r.plan, r.rank) for r, c in zip(ranks, columns)]
    for r, p in zip(ranks, planes):
        unpack_backward(p, r.plan, r.rank, [sends[j][r.rank] for j in range(len(ranks))])
    torch.cuda.synchronize()
    for r, f in zip(ranks, fields):
        r.backward(f)
