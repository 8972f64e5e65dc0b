"""The oracle against the reference's own kernel (CPU build), bit for bit.

tests/golden/*.npz were produced by tests/golden/make_golden.py from the reference
kernel source compiled for the CPU, on models shipped with the reference.  The
oracle, run in the reference's sequential ran3 mode from the same initial table,
must reproduce every per-photon exit record, every r-z buffer cell and the final
RNG state exactly.
"""
import glob
import os

import numpy as np
import pytest

import pyoracle as po
from golden.make_golden import arrays

GOLDEN = sorted(p for p in glob.glob(os.path.join(os.path.dirname(__file__), "golden", "model*.npz")))


def load_case(z):
    s = z["scalars"]
    tri, nrm, med = arrays(z)
    case = po.Case(tri=tri, nrm=nrm, med=med, nmuasg=z["nmuasg"], p_start=z["p_start"],
                   v_start=z["v_start"], ep0xyz=z["ep0xyz"], dimensions=z["dimensions"],
                   det_grid=z["det_grid"], fetal_id=int(s[0]), chance=float(s[1]),
                   w_threshold=float(s[2]), factor=float(s[3]))
    return case, int(s[4]), int(s[6])


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_oracle_reproduces_reference_kernel(oracle_lib, path):
    z = np.load(path)
    case, n, pad = load_case(z)
    r = po.run(case, n, rng_mode=po.RNG_RAN3_SHARED,
               ran3_state=(z["ran3_state0"], z["ran3_inext0"]), exit_records=True, rz_ref_pad=pad)
    want = z["exit_rec"]
    same = np.all(r.exit_rec.view(np.uint32) == want.view(np.uint32), axis=1)
    assert same.all(), f"first differing photon {np.argmin(same)}: {r.exit_rec[np.argmin(same)]} vs {want[np.argmin(same)]}"
    cells = np.nonzero(np.any(r.rz_ref != 0, axis=1))[0]
    assert np.array_equal(cells - pad, z["rz_cells"])
    assert np.array_equal(r.rz_ref[cells].view(np.uint32), z["rz_vals"].view(np.uint32))
    assert np.array_equal(r.ran3_state.view(np.uint32), z["ran3_state1"].view(np.uint32))
    assert np.array_equal(r.ran3_inext, z["ran3_inext1"])
    assert r.counters["rz_drop"] == 0      # no reference index fell outside the padded buffer


@pytest.mark.skipif(not po.ref_available(), reason="reference kernel build (oracle/_ref) not present")
@pytest.mark.parametrize("path", GOLDEN[:2], ids=[os.path.basename(p)[:-4] for p in GOLDEN[:2]])
def test_oracle_matches_reference_other_seeds(oracle_lib, path):
    """Live comparison with the compiled reference for seeds not in the fixtures."""
    z = np.load(path)
    case, _, pad = load_case(z)
    for seed in (5, 99):
        rec, rz, st, ix = po.ref_run(case, 400, ran3_seed=seed, rz_pad=pad)
        st0, ix0 = po.ref_ran3_state(seed)
        r = po.run(case, 400, rng_mode=po.RNG_RAN3_SHARED, ran3_state=(st0, ix0), exit_records=True,
                   rz_ref_pad=pad)
        assert np.array_equal(r.exit_rec.view(np.uint32), rec.view(np.uint32))
        assert np.array_equal(r.rz_ref.view(np.uint32), rz.view(np.uint32))
        assert np.array_equal(r.ran3_state.view(np.uint32), st.view(np.uint32))


@pytest.mark.skipif(not po.ref_available(), reason="reference kernel build (oracle/_ref) not present")
def test_find_triangle_matches_reference(oracle_lib):
    z = np.load([p for p in GOLDEN if p.endswith("model4_planar.npz")][0])
    tri = np.ascontiguousarray(z["tri"], np.float32)
    rng = np.random.default_rng(3)
    R, L = po.ref(), po.lib()
    for _ in range(2000):
        p = rng.uniform(-20, 20, 3).astype(np.float32)
        v = rng.normal(size=3)
        v = (v / np.linalg.norm(v)).astype(np.float32)
        ref_tri = int(rng.integers(-1, tri.shape[0]))
        t1 = np.zeros(1, np.float32)
        t2 = np.zeros(1, np.float32)
        a = R.clref_find_triangle(tri.shape[0], po.fptr(tri.ravel()), ref_tri, po.fptr(p), po.fptr(v), po.fptr(t1))
        b = L.lpo_find_triangle(po.fptr(tri.ravel()), tri.shape[0], ref_tri, po.fptr(p), po.fptr(v), po.fptr(t2))
        assert a == b and t1.view(np.uint32)[0] == t2.view(np.uint32)[0]
