"""Multi-rank path on the CPU: photon-range sharding and the integer all-reduce of tallies.

Ranks run as world_size-2 (and 3) gloo process groups.  Each rank traces its share of the
photon range with the oracle (the per-photon Philox streams the CUDA kernel uses), sums
the tallies with lightpropagation_b200.sharding, and rank 0 compares the sum with one
oracle run over the whole range.  The bar is equality bit for bit: integer tallies and
photon-indexed random streams make the split invisible.  On GPUs the same helpers run
over NCCL; that needs more than one GPU and is not exercised here."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import po, to_case
from lightpropagation_b200 import sharding, workloads

KEYS = ("sft", "rtd", "rz", "vox", "rbins", "region", "det")


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _as_dict(r):
    return {k: getattr(r, k) for k in KEYS} | {"counters": r.counters}


def _case(kind):
    if kind == "slab":
        return to_case(workloads.plain_slab()), workloads.plain_slab().compat
    w = workloads.curved_abdomen(freq=6)
    return to_case(w), w.compat


def _worker(rank, world, port, kind, n, first, out_dir):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"], os.environ["MASTER_PORT"] = "127.0.0.1", str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        case, compat = _case(kind)
        f, k = sharding.photon_range(n, rank, world, first)
        part = po.run(case, k, first=f, compat=compat, seed=77, nthreads=1)
        d = _as_dict(part)
        d["grad"] = part.grad.ravel()            # FP64 differentiation sums, reduced as float64
        total = sharding.reduce_host_tallies(d)
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), f=f, k=k, grad=total["grad"],
                 counters=np.array([total["counters"][c] for c in sorted(total["counters"])], np.uint64),
                 **{key: total[key] for key in KEYS})
    finally:
        dist.destroy_process_group()


def _spawn(world, kind, n, first, tmp_path):
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, kind, n, first, str(tmp_path))) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(300)
    for p in procs:
        if p.is_alive():
            p.kill()
            p.join()
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    return [dict(np.load(tmp_path / f"rank{r}.npz")) for r in range(world)]


def test_photon_range_partitions_exactly():
    for n in (0, 1, 2, 7, 1000, 1001, 6400 * 3 + 5):
        for world in (1, 2, 3, 4, 8):
            for first in (0, 123456789012):
                parts = [sharding.photon_range(n, r, world, first) for r in range(world)]
                assert sum(k for _, k in parts) == n
                assert parts[0][0] == first
                for (f0, k0), (f1, _) in zip(parts, parts[1:]):
                    assert f0 + k0 == f1
                sizes = [k for _, k in parts]
                assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        sharding.photon_range(10, 2, 2)
    with pytest.raises(ValueError):
        sharding.photon_range(-1, 0, 1)


@pytest.mark.parametrize("world,kind,n,first", [(2, "slab", 1501, 0), (3, "slab", 1000, 5000),
                                                (2, "abdomen", 800, 17)])
def test_sharded_tallies_equal_one_rank(world, kind, n, first, tmp_path):
    outs = _spawn(world, kind, n, first, tmp_path)
    case, compat = _case(kind)
    full = po.run(case, n, first=first, compat=compat, seed=77, nthreads=0)
    ranges = sorted((int(o["f"]), int(o["k"])) for o in outs)
    assert ranges[0][0] == first and sum(k for _, k in ranges) == n
    want_counters = np.array([full.counters[c] for c in sorted(full.counters)], np.uint64)
    for o in outs:                      # every rank holds the full sum
        for key in KEYS:
            assert np.array_equal(o[key], getattr(full, key)), key
        assert np.array_equal(o["counters"], want_counters)
        # floating-point sums: equal to rounding
        assert np.allclose(o["grad"], full.grad.ravel(), rtol=1e-12, atol=0.0)
    if kind == "abdomen":
        assert full.det[:, 0].any() and full.grad.any()
    assert full.counters["photons"] == n
    assert full.region.sum() > 0


def _wrap_worker(rank, world, port, out_dir):
    import datetime
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"], os.environ["MASTER_PORT"] = "127.0.0.1", str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        big = np.array([2 ** 64 - 5, 2 ** 63 + 1, 3], np.uint64) if rank == 0 else np.array([7, 2 ** 63, 1], np.uint64)
        ts = [torch.from_numpy(big.view(np.int64).copy()), torch.arange(5, dtype=torch.int64) * (rank + 1)]
        sharding.allreduce_flat(ts)
        np.save(os.path.join(out_dir, f"w{rank}.npy"), np.concatenate([t.numpy().view(np.uint64) for t in ts]))
    finally:
        dist.destroy_process_group()


def test_allreduce_flat_is_uint64_addition(tmp_path):
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_wrap_worker, args=(r, 2, port, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs)
    want = np.array([(2 ** 64 - 5 + 7) % 2 ** 64, (2 ** 63 + 1 + 2 ** 63) % 2 ** 64, 4, 0, 3, 6, 9, 12], np.uint64)
    for r in range(2):
        assert np.array_equal(np.load(tmp_path / f"w{r}.npy"), want)
