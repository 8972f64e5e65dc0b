"""Photon-range sharding across ranks, and the one exchange step: a sum of tallies.

Photons are independent histories.  Rank r of W traces the contiguous photon-index
range ``photon_range(n, r, W, first)`` under the same Philox key, so the ranks together
trace exactly the photons that one GPU traces for ``[first, first + n)``: photon i draws
its random numbers from counter (i, event, stream) whichever rank runs it.  Every tally
is a uint64 fixed-point sum (2^32 per unit weight), and integer addition is associative
and commutative, so the tallies summed over ranks equal the single-GPU tallies bit for
bit.  That sum is the path's only collective: one all-reduce of one flat int64 buffer
per launch (NCCL over NVLink on GPUs, gloo on CPU for tests).  uint64 values travel as
int64; two's-complement addition wraps exactly like uint64 addition.  A differentiated
run adds the FP64 perturbation sums, reduced in a second, float64 all-reduce: those
agree with one GPU's to rounding, not bit for bit.

This replaces nothing in the reference, which runs on one OpenCL device
(CalculatePropagation.cpp:1389-1759); the photon loop it splits into 6400-photon
launches is split here across ranks instead.
"""
from __future__ import annotations

from typing import Dict, Iterable, List, Optional, Tuple

import numpy as np

TALLY_KEYS = ("sft", "rtd", "rz", "vox", "rbins", "region", "det")


def photon_range(n: int, rank: int, world: int, first: int = 0) -> Tuple[int, int]:
    """(first index, count) of rank's share of photons [first, first + n).  Shares are
    contiguous, in rank order, and differ in size by at most one photon."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} of world {world}")
    if n < 0 or first < 0:
        raise ValueError("negative photon range")
    base, extra = divmod(int(n), int(world))
    start = first + rank * base + min(rank, extra)
    return start, base + (1 if rank < extra else 0)


def allreduce_flat(tensors: List["object"], group=None) -> None:
    """Sum tensors over the process group in place with one all-reduce per dtype (int64
    tallies; float64 differentiation sums, if any): pack each dtype's tensors into a
    flat buffer on their device, reduce it, unpack."""
    import torch
    import torch.distributed as dist
    if not tensors:
        return
    for t in tensors:
        if t.dtype not in (torch.int64, torch.float64):
            raise TypeError("tallies are reduced as int64, differentiation sums as float64")
    for dt in (torch.int64, torch.float64):
        part = [t for t in tensors if t.dtype == dt]
        if not part:
            continue
        flat = torch.cat([t.reshape(-1) for t in part])
        dist.all_reduce(flat, op=dist.ReduceOp.SUM, group=group)
        off = 0
        for t in part:
            k = t.numel()
            t.view(-1).copy_(flat[off:off + k])
            off += k


def reduce_host_tallies(tallies: Dict[str, object], group=None) -> Dict[str, object]:
    """Sum host tallies (numpy uint64 arrays, the ``counters`` dict and, if present, the
    float64 ``grad`` differentiation sums) over the group.  Returns a new dict with the
    same keys and shapes; the inputs are not modified."""
    import torch
    keys = [k for k in TALLY_KEYS if k in tallies]
    arrays = [np.ascontiguousarray(tallies[k], np.uint64) for k in keys]
    names = sorted(tallies["counters"]) if "counters" in tallies else []
    cnt = np.array([tallies["counters"][k] for k in names], np.uint64)
    ts = [torch.from_numpy(a.view(np.int64).copy()) for a in arrays + [cnt]]
    grad = None
    if tallies.get("grad") is not None:
        grad = torch.from_numpy(np.array(tallies["grad"], np.float64, copy=True))
        ts.append(grad)
    allreduce_flat(ts, group)
    out = {k: t.numpy().view(np.uint64).reshape(a.shape) for k, a, t in zip(keys, arrays, ts)}
    if names:
        out["counters"] = {k: int(v) for k, v in zip(names, ts[len(arrays)].numpy().view(np.uint64))}
    if grad is not None:
        out["grad"] = grad.numpy()
    return out


class _DeviceArray:
    """A raw device pointer seen by torch through __cuda_array_interface__."""

    def __init__(self, ptr: int, count: int, typestr: str = "<i8"):
        self.__cuda_array_interface__ = {"shape": (int(count),), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 3}


def device_tally_tensors(sim, device: int) -> List["object"]:
    """The context's device tally buffers (and counters) as int64 torch tensors that alias
    them, plus the differentiation sums as one float64 tensor while differentiation is on;
    valid until the tally layout changes (lp_set_tally_grid / lp_set_extra_tallies) or
    differentiation is switched."""
    import torch
    d = sim.device_tallies()
    out = []
    for name in TALLY_KEYS + ("counters",):
        cnt = getattr(d, "n_" + name)
        if cnt > 0:
            out.append(torch.as_tensor(_DeviceArray(getattr(d, name), cnt), device=f"cuda:{device}"))
    if d.n_grad > 0:
        out.append(torch.as_tensor(_DeviceArray(d.grad, d.n_grad, "<f8"), device=f"cuda:{device}"))
    return out


def run_sharded(sim, n: int, first: int = 0, group=None, device: Optional[int] = None,
                tensors: Optional[Iterable["object"]] = None) -> None:
    """Trace this rank's share of photons [first, first + n) on its GPU into the zeroed
    tallies of `sim`, then sum the device tallies over the group in place (NCCL).
    Afterwards every rank's ``sim.tallies()`` holds the tallies of all n photons.
    `tensors` may pass the aliases from device_tally_tensors to skip re-querying them."""
    import torch
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    f, k = photon_range(n, rank, world, first)
    sim.run(k, f)
    dev = torch.cuda.current_device() if device is None else device
    ts = list(tensors) if tensors is not None else device_tally_tensors(sim, dev)
    with torch.cuda.device(dev):
        allreduce_flat(ts, group)
        torch.cuda.current_stream().synchronize()
