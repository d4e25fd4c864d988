"""One periodic mesh over several GPUs: slabs of cell layers and a halo exchange.

The reference partitions the triangulation over MPI ranks and refreshes the ghost values of
the solution before every residual (DGBase::assemble_residual, src/dg/dg_base.cpp:2742) and of
the auxiliary solution before the viscous face terms (src/dg/strong_dg.cpp:648). Here rank r
of W owns a slab of whole cell layers of the periodic cube (`slab_bounds`), the library packs
only the partition faces' data its neighbours read (ph_ctx_create_slab, ph_set_halo_exchange
in include/philip_b200.h), and `DistributedHalo` moves it with torch.distributed
point-to-point messages: one NCCL group per exchange on GPUs (stream-ordered: the transfer
waits on the context stream's packing and the context stream waits on the transfer before
unpacking, with the cells that read no ghost data computed in between), tagged gloo messages
on the CPU. The volume averages of a slab are its share of the mesh's: `global_integrals`
sums them over ranks (and takes the max wave speed).
"""
from __future__ import annotations

import ctypes
import sys
import traceback

from . import _lib


def slab_bounds(n: int, world: int, rank: int) -> tuple[int, int]:
    """(z_first, z_count) of rank's slab: the n layers split into world runs whose lengths
    differ by at most one, the longer ones first."""
    if not 1 <= world <= n:
        raise ValueError(f"{world} slabs of a mesh with {n} layers")
    base, extra = divmod(n, world)
    return rank * base + min(rank, extra), base + (1 if rank < extra else 0)


class _DeviceBytes:
    """A device allocation of the library seen as a torch uint8 tensor (no copy)."""

    def __init__(self, ptr: int, nbytes: int):
        self.__cuda_array_interface__ = {"shape": (nbytes,), "typestr": "|u1", "data": (ptr, False),
                                         "version": 3, "strides": None, "stream": None}


def _as_tensor(ptr: int, nbytes: int, device: str):
    import torch
    if device == "cpu":
        return torch.frombuffer((ctypes.c_uint8 * nbytes).from_address(ptr), dtype=torch.uint8)
    return torch.as_tensor(_DeviceBytes(ptr, nbytes), device=device)


class DistributedHalo:
    """ph_halo_fn over torch.distributed: at PH_HALO_BEGIN the downward pair (send_lo to the
    rank below, recv_hi from the rank above) then the upward pair (send_hi to the rank above,
    recv_lo from the rank below) are issued as one batch; at PH_HALO_END the context stream
    waits for them. The two pairs carry distinct tags and are issued in the same order on every
    rank, so they match also when the ranks below and above are the same (two ranks)."""

    def __init__(self, group=None, device: str = "cuda"):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.device = device
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        glob = (lambda r: dist.get_global_rank(group, r)) if group is not None else (lambda r: r)
        self.lo = glob((self.rank - 1) % self.world)
        self.hi = glob((self.rank + 1) % self.world)
        self._pending = None
        self.callback = _lib.HALO_FN(self._call)    # referenced for as long as the halo lives
        self.sum_callback = _lib.RANK_SUM_FN(self._sum)

    def _stream_ctx(self, stream):
        import contextlib
        import torch
        if self.device == "cpu":
            return contextlib.nullcontext()
        s = torch.cuda.ExternalStream(stream) if stream else torch.cuda.default_stream()
        return torch.cuda.stream(s)

    def begin(self, what: int, send_lo: int, send_hi: int, recv_lo: int, recv_hi: int, nbytes: int, stream=None):
        d = self.dist
        t = [_as_tensor(p, nbytes, self.device) for p in (send_lo, send_hi, recv_lo, recv_hi)]
        with self._stream_ctx(stream):
            ops = [d.P2POp(d.isend, t[0], self.lo, self.group, 2 * what),
                   d.P2POp(d.irecv, t[3], self.hi, self.group, 2 * what),
                   d.P2POp(d.isend, t[1], self.hi, self.group, 2 * what + 1),
                   d.P2POp(d.irecv, t[2], self.lo, self.group, 2 * what + 1)]
            self._pending = d.batch_isend_irecv(ops)

    def end(self, stream=None):
        reqs, self._pending = self._pending, None
        with self._stream_ctx(stream):
            for r in reqs or ():
                r.wait()

    def _call(self, user, what, phase, send_lo, send_hi, recv_lo, recv_hi, nbytes, stream):
        try:
            if phase == _lib.PH_HALO_BEGIN:
                self.begin(what, send_lo, send_hi, recv_lo, recv_hi, nbytes, stream)
            else:
                self.end(stream)
            return 0
        except Exception:   # reported to the library as a failed exchange
            traceback.print_exc(file=sys.stderr)
            return 1

    def sum(self, values):
        """values summed over the ranks (all-reduce of a float64 vector), as a list."""
        import torch
        t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM, group=self.group)
        return t.cpu().tolist()

    def _sum(self, user, values, count):   # ph_rank_sum_fn
        try:
            out = self.sum([values[i] for i in range(count)])
            for i in range(count):
                values[i] = out[i]
            return 0
        except Exception:
            traceback.print_exc(file=sys.stderr)
            return 1


class LoopbackHalo:
    """ph_halo_fn of a slab that owns every layer (one rank): its lower ghost layer is its own
    last layer and its upper ghost its own first, so recv_lo <- send_hi and recv_hi <- send_lo,
    two device copies on the context stream (no host synchronisation)."""

    def __init__(self, device: str = "cuda"):
        self.device = device
        self.callback = _lib.HALO_FN(self._call)
        self.sum_callback = _lib.RANK_SUM_FN(lambda user, values, count: 0)   # one rank: its own sum

    def _call(self, user, what, phase, send_lo, send_hi, recv_lo, recv_hi, nbytes, stream):
        try:
            if phase == _lib.PH_HALO_BEGIN:
                import contextlib
                import torch
                ctx = contextlib.nullcontext() if self.device == "cpu" else torch.cuda.stream(
                    torch.cuda.ExternalStream(stream) if stream else torch.cuda.default_stream())
                with ctx:
                    _as_tensor(recv_lo, nbytes, self.device).copy_(_as_tensor(send_hi, nbytes, self.device))
                    _as_tensor(recv_hi, nbytes, self.device).copy_(_as_tensor(send_lo, nbytes, self.device))
            return 0
        except Exception:
            traceback.print_exc(file=sys.stderr)
            return 1


def global_integrals(local, dist=None, device: str = "cpu"):
    """The mesh's ph_integrals values from every slab's: the three volume averages summed,
    the wave speed maximised."""
    import torch
    v = torch.tensor([float(x) for x in local], dtype=torch.float64, device=device)
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return v.tolist()
    s = v[:3].clone()
    m = v[3:].clone()
    dist.all_reduce(s, op=dist.ReduceOp.SUM)
    dist.all_reduce(m, op=dist.ReduceOp.MAX)
    return s.tolist() + m.tolist()
