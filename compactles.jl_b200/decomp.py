"""One rank of a decomposed grid: the reference's Decomp (src/decomposition.jl:
73-140) and the three points where its step calls MPI, for
`Solver(desc, decomp=..., exchange=...)` (cles_solver_create_decomposed).

    dc = Decomp(desc.n_global, dims=(1, 1, 4), coords=(0, 0, r), rank=r)
    ex = TorchExchange(dc)                       # one process per GPU, NCCL
    S = Solver(desc, ctx, decomp=dc, exchange=ex)
    S.set_state(dc.block(Q_global_interior), layout="interior")
    S.run(tfinal)

Ranks are numbered x fastest: rank = c0 + d0 (c1 + d1 c2) for coordinates
(c0, c1, c2) in a process grid of dims (d0, d1, d2).

`LocalGroup` runs every rank of a process grid inside one process, one host
thread per rank (its solver on its own stream): the library's in-process
exchange (cles_local_group_*).  `TorchExchange` binds the callbacks to
torch.distributed: NCCL point-to-point sends and receives for the halos,
all-gathers on the per-dimension sub-groups for the interface values and an
all-reduce for max_rate, all ordered on the solver's stream; over gloo it
moves host buffers (the CPU tests of the exchange logic).
"""
import ctypes as C

import numpy as np

from . import abi
from .api import _check, lib


def local_range(N, P, r):
    """local_range (src/decomposition.jl:73-78): rank r's (count, offset) of N points over P."""
    base, rem = divmod(int(N), int(P))
    return base + (1 if r < rem else 0), r * base + min(r, rem)


def coords_of(rank, dims):
    d0, d1, _ = dims
    return (rank % d0, (rank // d0) % d1, rank // (d0 * d1))


def rank_of(coords, dims):
    return coords[0] + dims[0] * (coords[1] + dims[1] * coords[2])


class Decomp:
    """This rank's place in a process grid over the global extents n_global."""

    def __init__(self, n_global, dims, coords, rank=None):
        self.n_global = tuple(int(v) for v in n_global)
        self.dims = tuple(int(v) for v in dims)
        self.coords = tuple(int(v) for v in coords)
        self.rank = rank_of(self.coords, self.dims) if rank is None else int(rank)
        rng = [local_range(self.n_global[k], self.dims[k], self.coords[k]) for k in range(3)]
        self.n_local = tuple(r[0] for r in rng)
        self.offset = tuple(r[1] for r in rng)

    @property
    def size(self):
        return self.dims[0] * self.dims[1] * self.dims[2]

    def struct(self):
        s = abi.cles_decomp()
        for k in range(3):
            s.dims[k] = self.dims[k]
            s.coords[k] = self.coords[k]
        s.rank = self.rank
        return s

    def slices(self):
        """This rank's block of a global interior array (z, y, x order)."""
        return tuple(slice(self.offset[k], self.offset[k] + self.n_local[k]) for k in (2, 1, 0))

    def block(self, Q_interior):
        """This rank's block of a global interior state (component, z, y, x)."""
        return np.ascontiguousarray(Q_interior[(slice(None),) + self.slices()])

    @staticmethod
    def all_ranks(n_global, dims):
        size = dims[0] * dims[1] * dims[2]
        return [Decomp(n_global, dims, coords_of(r, dims), r) for r in range(size)]


def assemble(decomps, blocks):
    """The global interior array from every rank's interior block."""
    d0 = decomps[0]
    nc = blocks[0].shape[0]
    out = np.zeros((nc,) + tuple(d0.n_global[k] for k in (2, 1, 0)), dtype=blocks[0].dtype)
    for dc, b in zip(decomps, blocks):
        out[(slice(None),) + dc.slices()] = b
    return out


class LocalGroup:
    """Every rank of a process grid in this process (cles_local_group_*):
    `exchange(coords)` is the exchange of the rank at coords.  A barrier not
    met within timeout_s seconds, or abort(), fails the pending calls with
    CLES_EXCHANGE on every rank."""

    def __init__(self, dims, timeout_s=60.0):
        self.dims = tuple(int(v) for v in dims)
        self.ptr = C.c_void_p()
        d = (C.c_int * 3)(*self.dims)
        _check(lib().cles_local_group_create(d, float(timeout_s), C.byref(self.ptr)))

    def exchange(self, coords):
        ex = _Struct()
        c = (C.c_int * 3)(*[int(v) for v in coords])
        _check(lib().cles_local_group_exchange(self.ptr, c, C.byref(ex.struct)))
        ex.owner = self   # the group must outlive the solvers that call into it
        return ex

    def abort(self):
        lib().cles_local_group_abort(self.ptr)

    def __del__(self):
        try:
            if self.ptr:
                lib().cles_local_group_destroy(self.ptr)
                self.ptr = None
        except Exception:
            pass


class _Struct:
    def __init__(self):
        self.struct = abi.cles_exchange()


class _CudaBytes:
    """A device byte range for torch.as_tensor (__cuda_array_interface__)."""

    def __init__(self, ptr, nbytes):
        self.__cuda_array_interface__ = {"shape": (int(nbytes),), "typestr": "|u1", "data": (int(ptr), False),
                                         "version": 3}


class TorchExchange:
    """cles_exchange over torch.distributed (one process per rank, the world
    laid out as the process grid).  Sub-groups along every split dimension
    are created here, collectively: every rank must construct its
    TorchExchange at the same point.  With the NCCL backend the buffers are
    device memory and every operation runs on the solver's stream; with gloo
    they are host memory."""

    TAG_UP, TAG_DOWN = 11, 12

    def __init__(self, decomp, group=None):
        import torch
        import torch.distributed as dist
        self.torch = torch
        self.dist = dist
        self.dc = decomp
        self.group = group
        if dist.get_world_size(group) != decomp.size:
            raise ValueError(f"process grid {decomp.dims} does not match communicator size "
                             f"{dist.get_world_size(group)}")
        self.device_buffers = dist.get_backend(group) == "nccl"
        self.errors = []
        # Cart_sub along each split dim: every line of ranks that differ only in
        # coordinate d, created in the same order on every rank
        self.sub = [None, None, None]
        dims = decomp.dims
        for d in range(3):
            if dims[d] == 1:
                continue
            others = [k for k in range(3) if k != d]
            for a in range(dims[others[1]]):
                for b in range(dims[others[0]]):
                    ranks = []
                    for r in range(dims[d]):
                        c = [0, 0, 0]
                        c[d], c[others[0]], c[others[1]] = r, b, a
                        ranks.append(self._global(rank_of(c, dims)))
                    g = dist.new_group(ranks)
                    if (decomp.coords[others[0]], decomp.coords[others[1]]) == (b, a):
                        self.sub[d] = g
        self._cb = (abi.HALO_FN(self._halo), abi.GATHER_FN(self._gather), abi.ALLREDUCE_FN(self._allreduce))
        self.struct = abi.cles_exchange(None, *self._cb)

    def _global(self, r):
        return r if self.group is None else self.dist.get_global_rank(self.group, r)

    def _peer(self, dim, coord):
        c = list(self.dc.coords)
        c[dim] = coord
        return self._global(rank_of(c, self.dc.dims))

    def _bytes(self, ptr, nbytes):
        torch = self.torch
        if nbytes == 0:
            return torch.empty(0, dtype=torch.uint8, device="cuda" if self.device_buffers else "cpu")
        if self.device_buffers:
            return torch.as_tensor(_CudaBytes(ptr, nbytes), device="cuda")
        arr = np.ctypeslib.as_array((C.c_uint8 * int(nbytes)).from_address(int(ptr)))
        return torch.from_numpy(arr)

    def _on_stream(self, stream):
        torch = self.torch
        if self.device_buffers and stream:
            return torch.cuda.stream(torch.cuda.ExternalStream(int(stream)))
        import contextlib
        return contextlib.nullcontext()

    # -- the three callbacks (exceptions are recorded and reported as failure) --
    def _halo(self, user, dim, prev, nxt, send_lo, send_hi, recv_lo, recv_hi, nbytes, stream):
        try:
            with self._on_stream(stream):
                self.halo(dim, prev, nxt, self._bytes(send_lo, nbytes), self._bytes(send_hi, nbytes),
                          self._bytes(recv_lo, nbytes), self._bytes(recv_hi, nbytes))
            return 0
        except Exception as e:   # noqa: BLE001 - reported through the status code
            self.errors.append(e)
            return 1

    def _gather(self, user, dim, local, allb, nbytes, stream):
        try:
            with self._on_stream(stream):
                self.gather(dim, self._bytes(local, nbytes), self._bytes(allb, nbytes * self.dc.dims[dim]))
            return 0
        except Exception as e:   # noqa: BLE001
            self.errors.append(e)
            return 1

    def _allreduce(self, user, op, vals, count):
        try:
            v = np.ctypeslib.as_array(vals, shape=(int(count),))
            v[:] = self.allreduce(op, v.copy())
            return 0
        except Exception as e:   # noqa: BLE001
            self.errors.append(e)
            return 1

    # -- the exchanges on tensors --
    def halo(self, dim, prev, nxt, send_lo, send_hi, recv_lo, recv_hi):
        """Sendrecv! with both neighbours along dim (src/halo.jl:143-194)."""
        dist = self.dist
        me = self.dc.coords[dim]
        ops, local = [], []
        if nxt >= 0:
            if nxt == me:
                local.append((recv_lo, send_hi))
            else:
                ops.append(dist.P2POp(dist.isend, send_hi, self._peer(dim, nxt), tag=self.TAG_UP))
        if prev >= 0:
            if prev == me:
                local.append((recv_hi, send_lo))
            else:
                ops.append(dist.P2POp(dist.isend, send_lo, self._peer(dim, prev), tag=self.TAG_DOWN))
        if prev >= 0 and prev != me:
            ops.append(dist.P2POp(dist.irecv, recv_lo, self._peer(dim, prev), tag=self.TAG_UP))
        if nxt >= 0 and nxt != me:
            ops.append(dist.P2POp(dist.irecv, recv_hi, self._peer(dim, nxt), tag=self.TAG_DOWN))
        for dst, src in local:
            dst.copy_(src)
        if ops:
            for w in dist.batch_isend_irecv(ops):
                w.wait()

    def gather(self, dim, local, allb):
        """Allgather! along dim in coordinate order (src/tridiag.jl:148)."""
        dist = self.dist
        g = self.sub[dim]
        n = self.dc.dims[dim]
        if n == 1:
            allb.copy_(local)
        elif self.device_buffers:
            dist.all_gather_into_tensor(allb, local, group=g)
        else:
            dist.all_gather(list(allb.view(n, -1).unbind(0)), local, group=g)

    def allreduce(self, op, vals):
        """Allreduce! of a few doubles over every rank (src/timestep.jl:173)."""
        torch, dist = self.torch, self.dist
        t = torch.tensor(vals, dtype=torch.float64, device="cuda" if self.device_buffers else "cpu")
        dist.all_reduce(t, op=dist.ReduceOp.MAX if op == abi.CLES_REDUCE_MAX else dist.ReduceOp.SUM,
                        group=self.group)
        return t.cpu().numpy()
