"""Transaction-sharded databases (include/tfim.h tfim_open_db_sharded).

Each shard holds a contiguous slice of the transactions; the library sums every partial
count (F1, row supports, each wave's b x d count matrix) over a group through an all-reduce
callback, so every shard sees the whole database's counts, takes the same search steps and
finds the same MFIs (integer sums: exact).  This is the multi-GPU design "transaction
sharding" for databases beyond one GPU's HBM; the reference itself runs on one GPU.

Two groups are provided:

* ``TorchGroup``: one process per GPU over ``torch.distributed`` (NCCL on NVLink / NVSwitch
  for device buffers).  The all-reduce is enqueued on the library's stream, so the count
  kernels, the collective and the threshold pass stay in stream order without a host sync.
* ``ThreadGroup``: several shards in one process, one host thread each, all on one GPU.
  The shards meet on the host (a barrier), one thread sums the partial buffers on the GPU,
  and every shard continues; no kernel waits on another.

Every shard must make the same library calls in the same order (the collectives match by
order); a shard that fails leaves the others to the group's timeout, after which their call
fails with TFIM_E_COMM.
"""
from __future__ import annotations

import sys
import threading
import traceback

import numpy as np

from . import _lib

_TYPESTR = {_lib.DT_I32: "<i4", _lib.DT_I64: "<i8"}


def shard_bounds(n: int, rank: int, world: int) -> tuple[int, int]:
    """Rows [lo, hi) of shard `rank` among `world` (contiguous, sizes differing by at most one)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a group of {world}")
    return n * rank // world, n * (rank + 1) // world


def shard_csr(offsets: np.ndarray, items: np.ndarray, rank: int, world: int) -> tuple[np.ndarray, np.ndarray]:
    """This shard's rows of a CSR transaction set, re-based to offset 0."""
    offsets = np.asarray(offsets, dtype=np.int64)
    lo, hi = shard_bounds(offsets.shape[0] - 1, rank, world)
    off = offsets[lo:hi + 1] - offsets[lo]
    return np.ascontiguousarray(off), np.ascontiguousarray(np.asarray(items, dtype=np.int32)[offsets[lo]:offsets[hi]])


class _CudaBuffer:
    """A device range described by the CUDA array interface (zero-copy view for torch)."""

    def __init__(self, ptr: int, count: int, dtype: int):
        self.__cuda_array_interface__ = {"shape": (int(count),), "typestr": _TYPESTR[dtype], "data": (int(ptr), False),
                                         "strides": None, "version": 3, "stream": None}


def device_view(ptr: int, count: int, dtype: int, device: int):
    """torch tensor aliasing `count` elements at device address `ptr` (raises if torch copied)."""
    import torch
    t = torch.as_tensor(_CudaBuffer(ptr, count, dtype), device=f"cuda:{device}")
    if t.data_ptr() != ptr:
        raise RuntimeError("the device buffer was copied instead of aliased")
    return t


class Group:
    """A member of a shard group: `rank` of `world`, and the all-reduce the library calls."""

    def __init__(self, rank: int, world: int):
        if world < 1 or not 0 <= rank < world:
            raise ValueError(f"rank {rank} outside a group of {world}")
        self.rank, self.world = int(rank), int(world)
        self.last_error = ""
        self._cfn = None

    def allreduce(self, ptr: int, count: int, dtype: int, op: int, stream: int) -> None:
        raise NotImplementedError

    def struct(self) -> _lib.Group:
        """The tfim_group handed to the library; this object keeps its callback alive."""
        def cb(buf, count, dtype, op, stream, user):
            try:
                self.allreduce(buf or 0, int(count), int(dtype), int(op), stream or 0)
                return 0
            except BaseException as e:   # the library turns a non-zero status into TFIM_E_COMM
                self.last_error = f"{type(e).__name__}: {e}"
                traceback.print_exc(file=sys.stderr)
                return 1
        self._cfn = _lib.ALLREDUCE_FN(cb)
        return _lib.Group(self.rank, self.world, self._cfn, None)


class TorchGroup(Group):
    """All-reduce over a torch.distributed process group (NCCL for CUDA buffers)."""

    def __init__(self, group=None, device: int = 0):
        import torch.distributed as dist
        super().__init__(dist.get_rank(group), dist.get_world_size(group))
        self.group, self.device = group, int(device)

    def allreduce(self, ptr, count, dtype, op, stream):
        import torch
        import torch.distributed as dist
        ops = {_lib.RED_SUM: dist.ReduceOp.SUM, _lib.RED_MIN: dist.ReduceOp.MIN, _lib.RED_MAX: dist.ReduceOp.MAX}
        t = device_view(ptr, count, dtype, self.device)
        s = torch.cuda.ExternalStream(stream, device=self.device) if stream else torch.cuda.current_stream(self.device)
        with torch.cuda.stream(s):
            dist.all_reduce(t, op=ops[op], group=self.group)


class ThreadGroup:
    """`world` shards in one process, one host thread each, all on one GPU (`device`).

    Every shard's context must be opened on `device`: the reduction views every shard's
    buffer as memory of that device.  ``run(fn)`` calls ``fn(member)`` in one thread per shard and returns the results in rank
    order; ``member.allreduce`` waits (on the host, up to `timeout` seconds) for every shard's
    partial buffer, sums them on the GPU into every buffer, and returns."""

    def __init__(self, world: int, device: int = 0, timeout: float = 120.0):
        self.world, self.device = int(world), int(device)
        self._barrier = threading.Barrier(self.world, timeout=timeout)
        self._slots = [None] * self.world
        self._error = None
        self.members = [_ThreadMember(self, r) for r in range(self.world)]

    def _allreduce(self, rank, ptr, count, dtype, op, stream):
        import torch
        if stream:
            torch.cuda.ExternalStream(stream, device=self.device).synchronize()
        else:
            torch.cuda.synchronize(self.device)
        self._slots[rank] = (ptr, count, dtype, op)
        self._barrier.wait()
        if rank == 0:
            try:
                kinds = {(c, d, o) for _, c, d, o in self._slots}
                if len(kinds) != 1:
                    raise RuntimeError(f"shards disagree on the collective (count, dtype, op): {sorted(kinds)}")
                with torch.cuda.device(self.device):
                    views = [device_view(p, c, d, self.device) for p, c, d, _ in self._slots]
                    acc = views[0].clone()
                    for v in views[1:]:
                        acc = acc + v if op == _lib.RED_SUM else torch.minimum(acc, v) if op == _lib.RED_MIN \
                            else torch.maximum(acc, v)
                    for v in views:
                        v.copy_(acc)
                    torch.cuda.synchronize(self.device)
                self._error = None
            except BaseException as e:
                self._error = e
        self._barrier.wait()
        if self._error is not None:
            raise RuntimeError(f"shard group all-reduce failed: {self._error}")

    def run(self, fn):
        """Results of fn(member) per shard; the first failure (in time) is re-raised.  A failed
        run leaves the group broken: make a new ThreadGroup for the next one."""
        out = [None] * self.world
        errs = []
        lock = threading.Lock()

        def body(r):
            try:
                out[r] = fn(self.members[r])
            except BaseException as e:
                with lock:
                    errs.append(e)
                self._barrier.abort()   # release the other shards from a pending all-reduce
        ts = [threading.Thread(target=body, args=(r,)) for r in range(self.world)]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
        if errs:
            raise errs[0]
        return out


class _ThreadMember(Group):
    def __init__(self, g: ThreadGroup, rank: int):
        super().__init__(rank, g.world)
        self._g = g

    def allreduce(self, ptr, count, dtype, op, stream):
        self._g._allreduce(self.rank, ptr, count, dtype, op, stream)
