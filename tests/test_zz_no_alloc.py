"""lp_run_noalloc: transport that allocates no device memory, against lp_run.

Some callers cannot let a library call cudaMalloc: an application that hands out device
memory from its own fixed arena, or code that cannot afford the device-wide
synchronisation that cudaFree implies.  lp_run_noalloc serves them: the caller owns every input and
output buffer, and the entry point keeps its scratch in a static device array.

Here the test plays that caller: it allocates the mesh and the output tallies itself
(torch tensors), calls lp_run_noalloc through the C ABI twice in a row, and requires
both results to equal those of lp_run in reference-arithmetic mode for the same seed and
photon range.  The tolerance is the one the determinism tests use: integer tallies,
equal bit for bit.  This file is collected last so that a failure here comes after
every other test has run."""
import ctypes as C

import numpy as np
import pytest

from lightpropagation_b200 import Simulation, _native, workloads

pytestmark = pytest.mark.gpu

KEYS = ("sft", "rtd", "rz", "region")


def _args(w, seed, n, tri, nrm, med, nm, out):
    a = _native.NoAllocArgs()
    a.tri, a.nrm, a.med, a.n_tri = tri.data_ptr(), nrm.data_ptr(), med.data_ptr(), w.n_tri
    a.nmuasg, a.n_media = _native.fptr(nm), w.nmuasg.shape[0]
    a.p_start[:] = [float(x) for x in w.p_start]
    a.v_start[:] = [float(x) for x in w.v_start]
    a.ep0xyz[:] = [float(x) for x in w.ep0xyz]
    a.fiber_radius = w.fiber_radius
    a.fiber_cos_max = w.src_cos_max if (w.fiber_radius > 0 or w.fiber_na > 0) else 1.0
    a.dimensions[:] = [float(x) for x in w.dimensions]
    a.det_grid[:] = [float(x) for x in w.det_grid]
    a.fetal_id, a.chance, a.w_threshold, a.factor = w.fetal_id, w.chance, w.w_threshold, w.factor
    a.seed, a.compat, a.first, a.n_photons = seed, w.compat, 0, n
    a.sft, a.rtd, a.rz = out["sft"].data_ptr(), out["rtd"].data_ptr(), out["rz"].data_ptr()
    a.region, a.counters = out["region"].data_ptr(), out["counters"].data_ptr()
    return a


def regular(w, n, seed):
    with Simulation(0) as s:
        w.apply(s, seed=seed)
        s.set_arithmetic(True)
        s.zero()
        s.run(n)
        return s.tallies(), s.geometry()


@pytest.mark.parametrize("case", ["slab", "abdomen"])
def test_noalloc_equals_lp_run_twice(case):
    import torch

    w = workloads.plain_slab() if case == "slab" else workloads.curved_abdomen(freq=6)
    assert w.n_tri <= _native.NOALLOC_MAX_TRI
    n, seed = 20000, 91
    ref, g = regular(w, n, seed)

    dev = torch.device("cuda", 0)
    tri = torch.from_numpy(np.ascontiguousarray(w.tri, np.float32).ravel()).to(dev)
    nrm = torch.from_numpy(np.ascontiguousarray(w.nrm, np.float32).ravel()).to(dev)
    med = torch.from_numpy(np.ascontiguousarray(w.med, np.int32).ravel()).to(dev)
    nm = np.ascontiguousarray(w.nmuasg, np.float32).ravel()
    sizes = {"sft": g.sft_nx * g.sft_ny * 3, "rtd": g.dimR * g.dimAlpha * 3, "rz": g.rz_nr * g.rz_nz * 2,
             "region": w.nmuasg.shape[0], "counters": 16}
    out = {k: torch.zeros(v, dtype=torch.int64, device=dev) for k, v in sizes.items()}

    a = _args(w, seed, n, tri, nrm, med, nm, out)

    L = _native.lib()
    stream = torch.cuda.current_stream(dev).cuda_stream
    for call in range(2):
        for t in out.values():
            t.zero_()
        torch.cuda.synchronize(dev)
        rc = L.lp_run_noalloc(C.byref(a), C.c_void_p(stream))
        assert rc == 0, L.lp_last_error(None)
        torch.cuda.synchronize(dev)
        for k in KEYS:
            got = out[k].cpu().numpy().view(np.uint64)
            assert np.array_equal(got, ref[k].ravel()), (call, k)
        cnt = out["counters"].cpu().numpy().view(np.uint64)
        assert int(cnt[8]) == n, (call, cnt[8])
        assert int(cnt[0]) == ref["counters"]["scatter"] and int(cnt[1]) == ref["counters"]["boundary"]


def test_noalloc_rejects_sizes_beyond_the_limits():
    a = _native.NoAllocArgs()
    one = np.zeros(4, np.float32)
    a.tri = a.nrm = a.med = a.sft = a.rtd = a.rz = a.region = 1   # never dereferenced: rejected first
    a.nmuasg, a.n_media = _native.fptr(one), 1
    a.n_tri = _native.NOALLOC_MAX_TRI + 1
    L = _native.lib()
    assert L.lp_run_noalloc(C.byref(a), None) == 5
    assert b"4096" in L.lp_last_error(None)
    a.n_tri, a.n_media = 16, _native.NOALLOC_MAX_MEDIA + 1
    assert L.lp_run_noalloc(C.byref(a), None) == 5
    assert b"64" in L.lp_last_error(None)


def test_noalloc_rejects_bad_dimensions():
    """Non-finite or non-positive model dimensions and image extents of 2^20 cells or more
    are refused before anything touches the GPU (the kernel would index the caller's
    buffers with the extents)."""
    w = workloads.plain_slab()
    one = np.ascontiguousarray(w.nmuasg, np.float32).ravel()
    L = _native.lib()
    a = _native.NoAllocArgs()
    a.tri = a.nrm = a.med = a.sft = a.rtd = a.rz = a.region = 1   # never dereferenced: rejected first
    a.nmuasg, a.n_media, a.n_tri = _native.fptr(one), w.nmuasg.shape[0], 16
    a.det_grid[:] = [1.0] * 6
    a.chance, a.factor, a.w_threshold, a.n_photons = 0.1, 1.0, 1e-4, 10
    for dims, code in (([float("nan"), 10.0, 10.0], 1), ([10.0, float("inf"), 10.0], 1), ([10.0, 10.0, 0.0], 1),
                       ([10.0, -5.0, 10.0], 1), ([10.0, 10.0, 3e6], 5)):
        a.dimensions[:] = dims
        assert L.lp_run_noalloc(C.byref(a), None) == code, dims
    a.dimensions[:] = [10.0, 10.0, 10.0]
    a.det_grid[:] = [1.0, 1.0, 1.0, 1.0, 1.0, 1e-6]
    assert L.lp_run_noalloc(C.byref(a), None) == 5
    a.det_grid[:] = [1.0] * 6
    a.n_photons = 2 ** 31 + 1                                     # one call indexes photons with 32 bits
    assert L.lp_run_noalloc(C.byref(a), None) == 5


def test_noalloc_refuses_out_of_range_region_ids():
    """The regular path refuses a region id outside [0, n_media) (lp_set_mesh a negative
    one, lp_run one past the media table); the device-side check of lp_run_noalloc makes
    the same mesh trace no photon and reports the bad triangles in
    counters[LP_C_BAD_INPUT].  A following call with a valid mesh traces normally."""
    import torch

    w = workloads.plain_slab()
    bad = np.ascontiguousarray(w.med, np.int32).copy()
    bad[3, 1] = w.nmuasg.shape[0]          # one past the last region
    bad[7, 0] = -1
    with Simulation(0) as s:
        with pytest.raises(Exception):
            s.set_mesh(w.tri, w.nrm, bad)
    _, g = regular(w, 10, 5)
    dev = torch.device("cuda", 0)
    tri = torch.from_numpy(np.ascontiguousarray(w.tri, np.float32).ravel()).to(dev)
    nrm = torch.from_numpy(np.ascontiguousarray(w.nrm, np.float32).ravel()).to(dev)
    med_bad = torch.from_numpy(bad.ravel()).to(dev)
    med_ok = torch.from_numpy(np.ascontiguousarray(w.med, np.int32).ravel()).to(dev)
    nm = np.ascontiguousarray(w.nmuasg, np.float32).ravel()
    sizes = {"sft": g.sft_nx * g.sft_ny * 3, "rtd": g.dimR * g.dimAlpha * 3, "rz": g.rz_nr * g.rz_nz * 2,
             "region": w.nmuasg.shape[0], "counters": 16}
    out = {k: torch.zeros(v, dtype=torch.int64, device=dev) for k, v in sizes.items()}
    L = _native.lib()
    stream = torch.cuda.current_stream(dev).cuda_stream
    a = _args(w, 3, 5000, tri, nrm, med_bad, nm, out)
    assert L.lp_run_noalloc(C.byref(a), C.c_void_p(stream)) == 0
    torch.cuda.synchronize(dev)
    cnt = out["counters"].cpu().numpy().view(np.uint64)
    assert int(cnt[_native.COUNTER_NAMES.index("bad_input")]) == 2
    assert int(cnt[_native.COUNTER_NAMES.index("photons")]) == 0
    assert not out["sft"].any() and not out["region"].any()
    a = _args(w, 3, 5000, tri, nrm, med_ok, nm, out)
    assert L.lp_run_noalloc(C.byref(a), C.c_void_p(stream)) == 0
    torch.cuda.synchronize(dev)
    cnt = out["counters"].cpu().numpy().view(np.uint64)
    assert int(cnt[_native.COUNTER_NAMES.index("bad_input")]) == 0
    assert int(cnt[_native.COUNTER_NAMES.index("photons")]) == 5000
