"""apply_along! on a line split across ranks: the reference's Decomp with P > 1
ranks along one dimension (src/decomposition.jl:80-122), one process per GPU.

The arithmetic runs in libcles.so (cles_split_* in cles.h); this module moves
the data between ranks with torch.distributed at the two points the
reference calls MPI:

* the halo exchange of the M planes next to each rank interface
  (exchange_halos!, src/halo.jl:143-194: Sendrecv! with both neighbours);
* the all-gather of every rank's local heads and tails
  (solve_lines!, src/tridiag.jl:148; src/banded.jl:190).

With the NCCL backend the buffers are device tensors on the GPU's current
stream; the library context must be ordered on that stream
(`Context(device, stream=torch.cuda.current_stream().cuda_stream)`), which
`SplitPlan` does by default.  The exchange itself is backend-neutral:
`LineExchange` also runs over gloo with CPU tensors.

    plan = SplitPlan(scheme, n_local, dim, h, n_global, ranks, rank, periodic)
    ex = LineExchange(plan.prev, plan.next, group)
    split_apply_along(out, plan, f, ex)     # out, f: padded CUDA tensors
"""
import ctypes as C

from . import abi
from .api import _check, lib

# message tags: planes travelling to the next rank / to the previous rank
TAG_UP = 1
TAG_DOWN = 2


class LineExchange:
    """Halo and interface exchange of a split line over a process group.

    `prev` and `next` are the neighbouring ranks' coordinates along the split
    dimension (None at a closed end); they are ranks of `group` (the
    sub-communicator along the dimension, the whole world by default)."""

    def __init__(self, prev, next, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.prev = prev
        self.next = next
        self.rank = dist.get_rank(group)
        self.size = dist.get_world_size(group)

    def _peer(self, r):
        if self.group is None:
            return r
        return self.dist.get_global_rank(self.group, r)

    def halo(self, send_lo, send_hi, recv_lo, recv_hi):
        """Sendrecv! with both neighbours: recv_lo <- prev's send_hi,
        recv_hi <- next's send_lo.  A rank that is its own neighbour (one
        periodic rank) copies."""
        dist = self.dist
        ops = []
        local = []
        # sends first, each direction with its own tag; a receive is posted in
        # the order its peer posts the matching send (two messages to one peer
        # when two ranks wrap around each other)
        if self.next is not None:
            if self.next == self.rank:
                local.append((recv_lo, send_hi))
            else:
                ops.append(dist.P2POp(dist.isend, send_hi, self._peer(self.next), self.group, TAG_UP))
        if self.prev is not None:
            if self.prev == self.rank:
                local.append((recv_hi, send_lo))
            else:
                ops.append(dist.P2POp(dist.isend, send_lo, self._peer(self.prev), self.group, TAG_DOWN))
        if self.prev is not None and self.prev != self.rank:
            ops.append(dist.P2POp(dist.irecv, recv_lo, self._peer(self.prev), self.group, TAG_UP))
        if self.next is not None and self.next != self.rank:
            ops.append(dist.P2POp(dist.irecv, recv_hi, self._peer(self.next), self.group, TAG_DOWN))
        for dst, src in local:
            dst.copy_(src)
        if ops:
            for w in dist.batch_isend_irecv(ops):
                w.wait()

    def gather(self, iface, iface_all):
        """Allgather! of the local heads and tails, rank-major into iface_all
        (shape (ranks,) + iface.shape)."""
        dist = self.dist
        if self.size == 1:
            iface_all[0].copy_(iface)
            return
        if dist.get_backend(self.group) == "nccl":
            dist.all_gather_into_tensor(iface_all, iface.unsqueeze(0), group=self.group)
        else:
            dist.all_gather(list(iface_all.unbind(0)), iface, group=self.group)


class SplitPlan:
    """plan_direction on a dimension split across ranks (cles_split_plan_create).

    n_local: this rank's interior extents (x, y, z); dim: 1-based split
    dimension; n_global: the global extent along it; rank / ranks: this
    rank's coordinate and the number of ranks along it."""

    def __init__(self, scheme, n_local, dim, h, n_global, ranks, rank, periodic, n_halo=4, dtype="f64", ctx=None):
        from .api import Context
        if ctx is None:
            import torch
            ctx = Context(torch.cuda.current_device(), stream=torch.cuda.current_stream().cuda_stream)
        self.ctx = ctx
        self.dtype = abi.CLES_F64 if dtype in ("f64", "float64") else abi.CLES_F32
        d = abi.cles_split_desc()
        for k in range(3):
            d.n_local[k] = int(n_local[k])
        d.n_halo = int(n_halo)
        d.dim = int(dim)
        d.n_global = int(n_global)
        d.ranks = int(ranks)
        d.rank = int(rank)
        d.periodic = int(bool(periodic))
        self.desc = d
        self.n_local = tuple(int(v) for v in n_local)
        self.n_halo = int(n_halo)
        self.dim = int(dim)
        self.ptr = C.c_void_p()
        _check(lib().cles_split_plan_create(self.ctx.ptr, C.byref(d), C.byref(scheme), float(h), self.dtype,
                                            C.byref(self.ptr)))
        info = abi.cles_split_info()
        _check(lib().cles_split_plan_info(self.ptr, C.byref(info)))
        self.info = info
        self.prev = info.prev if info.prev >= 0 else None
        self.next = info.next if info.next >= 0 else None

    def shape(self):
        """Padded field shape (z, y, x)."""
        return tuple(n + 2 * self.n_halo if n > 1 else 1 for n in reversed(self.n_local))

    def buffers(self, count, device):
        """Exchange buffers for `count` fields: send/recv halos and the
        local / gathered interface values."""
        import torch
        dt = torch.float64 if self.dtype == abi.CLES_F64 else torch.float32
        he, ie = count * self.info.halo_elems, count * self.info.iface_elems
        z = lambda *s: torch.zeros(*s, dtype=dt, device=device)
        return dict(send_lo=z(he), send_hi=z(he), recv_lo=z(he), recv_hi=z(he), iface=z(ie),
                    iface_all=z(self.info.ranks, ie))

    def _stride(self, count, field_stride):
        return int(field_stride) if field_stride is not None else int(self.info.field_elems)

    def pack(self, f, bufs, count=1, field_stride=None):
        _check(lib().cles_split_halo_pack(self.ptr, C.c_void_p(f.data_ptr()), C.c_void_p(bufs["send_lo"].data_ptr()),
                                          C.c_void_p(bufs["send_hi"].data_ptr()), int(count),
                                          self._stride(count, field_stride)))

    def unpack(self, bufs, f, count=1, field_stride=None):
        _check(lib().cles_split_halo_unpack(self.ptr, C.c_void_p(bufs["recv_lo"].data_ptr()),
                                            C.c_void_p(bufs["recv_hi"].data_ptr()), C.c_void_p(f.data_ptr()),
                                            int(count), self._stride(count, field_stride)))

    def begin(self, f, out, bufs, count=1, field_stride=None):
        _check(lib().cles_split_apply_begin(self.ptr, C.c_void_p(f.data_ptr()), C.c_void_p(out.data_ptr()),
                                            C.c_void_p(bufs["iface"].data_ptr()), int(count),
                                            self._stride(count, field_stride)))

    def end(self, bufs, out, count=1, field_stride=None):
        _check(lib().cles_split_apply_end(self.ptr, C.c_void_p(bufs["iface_all"].data_ptr()),
                                          C.c_void_p(out.data_ptr()), int(count), self._stride(count, field_stride)))

    def __del__(self):
        try:
            if self.ptr:
                lib().cles_split_plan_destroy(self.ptr)
                self.ptr = None
        except Exception:
            pass


def exchange_halos(plan, f, exchange, bufs=None, count=1, field_stride=None):
    """exchange_halos! along the split dimension (src/halo.jl:143-194) for the
    planes the operator reads."""
    bufs = bufs or plan.buffers(count, f.device)
    plan.pack(f, bufs, count, field_stride)
    exchange.halo(bufs["send_lo"], bufs["send_hi"], bufs["recv_lo"], bufs["recv_hi"])
    plan.unpack(bufs, f, count, field_stride)
    return bufs


def split_apply_along(out, plan, f, exchange, bufs=None, count=1, field_stride=None, halos_current=False):
    """apply_along!(out, plan, f, decomp) on a split dimension: halo exchange
    (unless halos_current), local solve, interface all-gather, correction.
    Writes the interior of `out`; f's halo planes are overwritten."""
    bufs = bufs or plan.buffers(count, f.device)
    if not halos_current:
        exchange_halos(plan, f, exchange, bufs, count, field_stride)
    plan.begin(f, out, bufs, count, field_stride)
    exchange.gather(bufs["iface"], bufs["iface_all"])
    plan.end(bufs, out, count, field_stride)
    return out
