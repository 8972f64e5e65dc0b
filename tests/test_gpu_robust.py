"""Host-side robustness of the CUDA path (marked gpu), each without faulting the GPU.

  * the per-photon step cap (the watchdog of a photon that would run on): the launch
    returns, and the photons it stopped are counted;
  * checkpoint and resume: photons [0, k) traced and saved, then resumed in a new
    context from the saved tallies, give one uninterrupted run's tallies bit for bit
    (the reference carries only its ran3 table between launches,
    CalculatePropagation.cpp:1213-1215);
  * an allocation that fails (injected on the host by lp_debug_fail_allocation) is
    reported as LP_ERR_NOMEM and leaves the context usable;
  * the NCCL reduction of run_sharded on one rank: the device-alias path of the
    multi-GPU code, integer tallies and FP64 differentiation sums;
  * the bounds-checked build (liblpcuda_debug.so, in place of compute-sanitizer, which
    this pool does not offer) counts no out-of-range index and changes no tally;
  * a photon range longer than 2^31 (the kernel indexes a launch's photons with 32 bits)
    runs as several launches with the tallies of the same range run as separate calls.
"""
import datetime
import os
import socket

import numpy as np
import pytest

import pyoracle as po
from conftest import to_case
from lightpropagation_b200 import Simulation, _native, sharding, workloads

pytestmark = pytest.mark.gpu

KEYS = ("sft", "rtd", "rz", "vox", "rbins", "region", "det")


def test_step_cap_stops_photons_and_counts_them():
    """With at most 5 steps per photon nearly every slab photon (about 2,600 scatter events
    each) is stopped; the GPU stops the same photons as the oracle with the same cap and
    common random numbers, and every photon is accounted for."""
    w = workloads.plain_slab()
    n = 20000
    with Simulation(0) as s:
        w.apply(s, seed=55)
        s.set_arithmetic(True)
        s.set_max_steps(5)
        s.zero()
        s.run(n)
        t = s.tallies()
    c = t["counters"]
    assert c["photons"] == n
    assert c["capped"] > 0.9 * n
    assert c["scatter"] + c["boundary"] <= 5 * n
    r = po.run(to_case(w), n, rng_mode=po.RNG_PHILOX, seed=55, compat=w.compat, max_steps=5)
    assert abs(c["capped"] - r.counters["capped"]) <= 0.002 * n, (c["capped"], r.counters["capped"])
    # a capped photon ends without an exit weight: only the photons that left within 5 steps score
    assert t["sft"][:, :, 0].sum() <= (n - c["capped"] + 1) * 2 ** 32


@pytest.mark.parametrize("case", ["slab", "abdomen_grad"])
def test_checkpoint_resume_is_bit_identical(case, tmp_path):
    w = workloads.plain_slab() if case == "slab" else workloads.curved_abdomen(freq=12)
    grad = case.endswith("grad")
    n, k = 40000, 15000
    with Simulation(0) as s:
        w.apply(s, seed=123)
        s.set_gradient(grad)
        s.zero()
        s.run(n, 0)
        full = s.checkpoint()
    with Simulation(0) as s:
        w.apply(s, seed=123)
        s.set_gradient(grad)
        s.zero()
        s.run(k, 0)
        saved = s.checkpoint()
    np.savez(tmp_path / "ckpt.npz", **saved)     # through a file, as a restart would
    loaded = dict(np.load(tmp_path / "ckpt.npz"))
    with Simulation(0) as s:                # a new context, as after a restart
        w.apply(s, seed=123)
        s.set_gradient(grad)
        s.zero()
        s.restore(loaded)
        s.run(n - k, k)
        resumed = s.checkpoint()
    for key in KEYS + ("counters",):
        assert np.array_equal(resumed[key], full[key]), key
    if grad:
        assert np.any(full["grad"])
        assert np.allclose(resumed["grad"], full["grad"], rtol=1e-12, atol=0.0)


def test_injected_allocation_failure_leaves_the_context_usable():
    """Every allocation a first run makes fails once in turn: the call returns
    LP_ERR_NOMEM, and after the injection is off the same context runs and gives the
    tallies of a clean context."""
    L = _native.lib()
    w = workloads.plain_slab()
    n = 5000
    with Simulation(0) as s:
        w.apply(s, seed=9)
        s.zero()
        s.run(n)
        want = s.tallies()
    failures = 0
    try:
        for k in range(64):
            with Simulation(0) as s:
                w.apply(s, seed=9)
                L.lp_debug_fail_allocation(k)
                try:
                    s.run(n)
                    s.tallies()
                    injected = False
                except _native.LPError as e:
                    assert e.code == 4, e
                    injected = True
                L.lp_debug_fail_allocation(-1)
                if not injected:
                    break
                failures += 1
                s.zero()
                s.run(n)
                got = s.tallies()
                for key in KEYS:
                    assert np.array_equal(got[key], want[key]), (k, key)
    finally:
        L.lp_debug_fail_allocation(-1)
    assert failures >= 10, failures


def _port():
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        return so.getsockname()[1]


def test_run_sharded_over_nccl_on_one_rank():
    """sharding.run_sharded with a one-rank NCCL group: the device tallies are aliased as
    torch tensors and all-reduced in place (integer tallies as int64, differentiation sums
    as float64); the result equals the plain run."""
    import torch
    import torch.distributed as dist
    w = workloads.curved_abdomen(freq=12)
    n = 50000
    with Simulation(0) as s:
        w.apply(s, seed=31)
        s.set_gradient(True)
        s.zero()
        s.run(n, 1000)
        want = s.checkpoint()
    os.environ["MASTER_ADDR"], os.environ["MASTER_PORT"] = "127.0.0.1", str(_port())
    os.environ.setdefault("NCCL_NVLS_ENABLE", "0")
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60),
                            device_id=torch.device("cuda", 0))
    try:
        with Simulation(0) as s:
            w.apply(s, seed=31)
            s.set_gradient(True)
            s.zero()
            s.run(0)
            ts = sharding.device_tally_tensors(s, 0)
            assert {t.dtype for t in ts} == {torch.int64, torch.float64}
            sharding.run_sharded(s, n, first=1000, tensors=ts)
            got = s.checkpoint()
            ts.clear()
    finally:
        dist.destroy_process_group()
    for key in KEYS + ("counters",):
        assert np.array_equal(got[key], want[key]), key
    # FP64 atomic sums: their order, and so their last bits, vary from run to run
    assert np.allclose(got["grad"], want["grad"], rtol=1e-12, atol=0.0)


_DEBUG_CHILD = r"""
import json, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
from lightpropagation_b200 import Simulation, _native, workloads
out = {"lib": _native.lib()._name}
for name, w in (("slab", workloads.plain_slab()), ("abdomen", workloads.curved_abdomen(freq=12))):
    for exact in (False, True):
        with Simulation(0) as s:
            w.apply(s, seed=71)
            s.set_arithmetic(exact)
            s.set_gradient(name == "abdomen")
            s.zero()
            s.run(20000)
            t = s.tallies()
        out[f"{name}-{int(exact)}"] = {k: np.asarray(t[k]).astype(np.uint64).tolist() for k in ("sft", "region", "det")}
        out[f"{name}-{int(exact)}"]["vox_sum"] = int(np.asarray(t["vox"], np.uint64).sum())
        out[f"{name}-{int(exact)}"]["counters"] = t["counters"]
print(json.dumps(out))
"""


def _run_child(debug):
    import json
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, LP_DEBUG_LIBRARY="1" if debug else "0")
    r = subprocess.run([sys.executable, "-c", _DEBUG_CHILD, root], capture_output=True, text=True, env=env,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_bounds_checked_build_finds_nothing_and_changes_nothing():
    """liblpcuda_debug.so checks every array index of the transport path (cell lists,
    BVH nodes, triangles, media, triangle attributes) and counts out-of-range accesses
    instead of making them.  On the slab and the abdomen, in both arithmetic modes and
    with differentiation, it counts none and gives the release build's tallies."""
    dbg, rel = _run_child(True), _run_child(False)
    assert dbg["lib"].endswith("liblpcuda_debug.so") and rel["lib"].endswith("liblpcuda.so")
    for key in (k for k in dbg if k != "lib"):
        assert dbg[key]["counters"]["bounds"] == 0, key
        for k in ("sft", "region", "det", "vox_sum"):
            assert dbg[key][k] == rel[key][k], (key, k)
        assert dbg[key]["counters"]["scatter"] == rel[key]["counters"]["scatter"]


def test_range_beyond_2_31_photons_runs_in_chunks():
    """2^31 + 1000 slab photons that end at their first roulette (weight threshold 1,
    survival chance 1e-6): one lp_run over the whole range (two launches inside) against
    lp_run over [0, 2^31) and then over the remaining 1000 photons on the same tallies."""
    w = workloads.plain_slab()
    w.w_threshold = 1.0
    w.chance = 1e-6
    n0 = 2 ** 31
    with Simulation(0) as s:
        w.apply(s, seed=5)
        s.zero()
        s.run(n0 + 1000, 0)
        one = s.tallies()
        s.zero()
        s.run(n0, 0)
        s.run(1000, n0)
        two = s.tallies()
    assert one["counters"]["photons"] == n0 + 1000
    for key in KEYS:
        assert np.array_equal(one[key], two[key]), key
    for k in ("scatter", "boundary", "roulette"):
        assert one["counters"][k] == two["counters"][k], k


@pytest.mark.parametrize("wname", ["slab", "abdomen"])
def test_tally_aggregation_changes_nothing(wname):
    """Warp-aggregated deposits (lanes that hit the same r-z cell or voxel are matched with
    __match_any_sync, their fixed-point values summed, one atomic per group) give the plain
    kernel's tallies bit for bit; the leader counter gives the match rate."""
    w = workloads.plain_slab() if wname == "slab" else workloads.curved_abdomen(freq=12)
    n = 200000
    out = []
    for agg in (False, True):
        with Simulation(0) as s:
            w.apply(s, seed=17)
            s.set_tally_aggregation(agg)
            s.zero()
            s.run(n)
            out.append(s.tallies())
    for key in KEYS:
        assert np.array_equal(out[0][key], out[1][key]), key
    c = out[1]["counters"]
    deposits = c["scatter"] - c["rz_drop"]
    assert 0 < c["agg_leaders"] <= deposits
    print(f"{wname}: r-z deposit groups {c['agg_leaders']} of {deposits} deposits, "
          f"match rate {1 - c['agg_leaders'] / deposits:.3f}")
