"""Batched transport on the GPU: every instance of one persistent launch must equal,
bit for bit, a single-instance lp_run on its context with its media and photon range
(integer tallies and event counters), for every launch configuration the autotuner can
pick, across CUDA-graph replays and instance updates, and with the large instances run
as transport launches of their own inside the graph.  Gradient sums are FP64 atomics
whose order differs between launches, so they are compared to 1e-9 relative."""
import numpy as np
import pytest

from lightpropagation_b200 import Batch, Instance, Simulation, workloads
from lightpropagation_b200.batch import config_table

pytestmark = pytest.mark.gpu

KEYS = ("sft", "rtd", "rz", "vox", "rbins", "region", "det")
COUNTERS = ("scatter", "boundary", "query", "roulette", "miss", "capped", "rz_drop", "vox_drop", "photons",
            "safe_skip", "bvh_query")


@pytest.fixture(scope="module")
def meshes2():
    a = workloads.curved_abdomen(freq=6)
    b = workloads.curved_abdomen(freq=6, head_depth=60.0, fat=(5.0, 20.0))
    return [a, b]


def _sim(w, seed=9):
    s = Simulation(0)
    w.apply(s, seed=seed)
    return s


def _instances(ws):
    rng = np.random.default_rng(4)
    out = []
    budgets = [3000, 1, 0, 4500, 777, 2500]
    for i, n in enumerate(budgets):
        ctx = i % 2
        nm = np.array(ws[ctx].nmuasg, np.float32)
        if i >= 2:
            nm[1:, 1] *= rng.uniform(0.8, 1.25, nm.shape[0] - 1).astype(np.float32)
            nm[1:, 2] *= rng.uniform(0.8, 1.25, nm.shape[0] - 1).astype(np.float32)
        out.append(Instance(context=ctx, nmuasg=nm, n_photons=n, first=int(rng.integers(0, 10 ** 9))))
    return out


def _single(ws, inst, grad=False):
    s = _sim(ws[inst.context])
    s.set_media(inst.nmuasg)
    s.set_gradient(grad)
    s.zero()
    s.run(inst.n_photons, inst.first)
    t = s.tallies()
    g = s.gradient() if grad else None
    s.close()
    return t, g


def _same(a, b, n_media):
    for k in KEYS:
        x, y = a[k], b[k]
        if k == "region":
            x, y = x[:n_media], y[:n_media]
        assert np.array_equal(x, y), k
    for k in COUNTERS:
        assert a["counters"][k] == b["counters"][k], k


def test_batch_equals_single_runs_for_every_config(meshes2):
    sims = [_sim(w) for w in meshes2]
    insts = _instances(meshes2)
    ref = [_single(meshes2, x)[0] for x in insts]
    with Batch(sims) as b:
        b.set_instances(insts)
        for k, cfg in enumerate(config_table()):
            b.set_config(k)
            b.run()
            for i, x in enumerate(insts):
                _same(b.tallies(i), ref[i], x.nmuasg.shape[0])
            assert b.tallies(0)["counters"]["photons"] == insts[0].n_photons
    for s in sims:
        s.close()


def test_graph_replay_and_instance_update(meshes2):
    sims = [_sim(w) for w in meshes2]
    insts = _instances(meshes2)
    with Batch(sims) as b:
        b.set_instances(insts)
        b.set_config(0)
        b.run()
        first = [b.tallies(i) for i in range(len(insts))]
        b.run()                                   # graph replay: same result
        for i, x in enumerate(insts):
            _same(b.tallies(i), first[i], x.nmuasg.shape[0])
        new = [Instance(x.context, x.nmuasg * np.float32([1, 1.1, 0.9, 1]), x.n_photons, x.first + 5) for x in insts]
        b.set_instances(new)                      # same count: the graph is reused with new parameters
        b.run()
        for i, x in enumerate(new):
            _same(b.tallies(i), _single(meshes2, x)[0], x.nmuasg.shape[0])
        sig, err = b.ring_signals()
        t0 = b.tallies(0)
        assert np.allclose(sig[0], t0["det"][:, 0] / 2.0 ** 32 / new[0].n_photons)
    for s in sims:
        s.close()


def test_batch_gradient_equals_single(meshes2):
    sims = [_sim(w) for w in meshes2]
    insts = _instances(meshes2)
    with Batch(sims) as b:
        b.set_instances(insts)
        b.set_gradient(True)
        b.set_config(2)
        b.run()
        for i, x in enumerate(insts):
            t, g = _single(meshes2, x, grad=True)
            _same(b.tallies(i), t, x.nmuasg.shape[0])
            bg = b.gradient(i)
            for k in ("signal", "d_mua", "d_mus"):
                assert np.allclose(bg[k], g[k], rtol=1e-9, atol=0), k
    for s in sims:
        s.close()


def test_large_instances_as_own_launches_equal_single_runs(meshes2):
    """With the plain threshold at 2000 photons the instances of 3000, 4500 and 2500
    photons run as transport launches of their own inside the graph, the rest in the batch
    launch: every instance still equals its single run, with and without differentiation,
    across a graph replay and an update of the instances."""
    sims = [_sim(w) for w in meshes2]
    insts = _instances(meshes2)
    with Batch(sims) as b:
        b.set_instances(insts)
        b.set_config(0)
        b.set_plain_threshold(2000)
        assert b.plain_count() == 3
        b.run()
        for i, x in enumerate(insts):
            _same(b.tallies(i), _single(meshes2, x)[0], x.nmuasg.shape[0])
        new = [Instance(x.context, x.nmuasg * np.float32([1, 1.05, 0.95, 1]), x.n_photons, x.first + 11)
               for x in insts]
        b.set_instances(new)
        b.run()
        b.run()
        for i, x in enumerate(new):
            _same(b.tallies(i), _single(meshes2, x)[0], x.nmuasg.shape[0])
        b.set_gradient(True)
        b.run()
        for i, x in enumerate(new):
            t, g = _single(meshes2, x, grad=True)
            _same(b.tallies(i), t, x.nmuasg.shape[0])
            bg = b.gradient(i)
            for k in ("signal", "d_mua", "d_mus"):
                assert np.allclose(bg[k], g[k], rtol=1e-9, atol=0), k
        b.set_plain_threshold(0)
        assert b.plain_count() == 0
    for s in sims:
        s.close()


def test_autotune_chooses_a_measured_config(meshes2):
    sims = [_sim(w) for w in meshes2]
    with Batch(sims) as b:
        b.set_instances(_instances(meshes2))
        best, ns = b.autotune(20000)
        assert 0 <= best < len(ns) and ns[best] > 0
        assert ns[best] == min(v for v in ns if v > 0)
        b.run()                                   # uses the chosen configuration
    for s in sims:
        s.close()


def test_batch_rejects_bad_instances(meshes2):
    sims = [_sim(w) for w in meshes2]
    with Batch(sims) as b:
        nm = np.array(meshes2[0].nmuasg, np.float32)
        with pytest.raises(Exception, match="context"):
            b.set_instances([Instance(context=5, nmuasg=nm, n_photons=10)])
        with pytest.raises(Exception, match="regions"):
            b.set_instances([Instance(context=0, nmuasg=np.tile(nm, (2, 1)), n_photons=10)])
    for s in sims:
        s.close()
