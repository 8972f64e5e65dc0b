"""The FP64 error oracle (oracle/lp_oracle64.c) on the CPU.

It restates the pinned FP32 oracle (itself bit-identical to the reference kernel, see
test_oracle_golden.py) in double precision, so it is checked against that oracle:

  * its tree search returns the brute-force scan's answer (index and distance) on rays
    that start on triangles, inside the meshes and outside them, with and without a
    bound;
  * with the same Philox numbers most photons follow the FP32 oracle's trajectory: their
    exit records agree to the FP32 rounding that separates the two;
  * with independent streams the scalar tallies agree within |z| < 3;
  * the committed statistics fixtures were made from the workloads as they are now.
"""
import os
import sys

import numpy as np
import pytest

import pyoracle as po
from conftest import to_case, z_scores
from lightpropagation_b200 import meshes, workloads

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
import fixture64 as fx  # noqa: E402

FIX = 2.0 ** 32


@pytest.mark.parametrize("mesh", ["slab", "abdomen", "soup"])
def test_tree_query_equals_brute_force(oracle_lib, mesh):
    rng = np.random.default_rng(5)
    if mesh == "slab":
        tri = meshes.layered_slab([2.0, 10.0, 30.0])[0]
        lo, hi = np.array([-55, -55, -5]), np.array([55, 55, 47])
    elif mesh == "abdomen":
        tri = meshes.curved_abdomen(freq=12)[0]
        lo, hi = np.array([-150, -120, -100]), np.array([150, 120, 100])
    else:
        c = rng.uniform(-20, 20, (2000, 1, 3))
        tri = (c + rng.normal(scale=3.0, size=(2000, 3, 3))).astype(np.float32).reshape(2000, 9)
        tri[1::7] = tri[0::7][: tri[1::7].shape[0]]          # exact duplicates: ties
        lo, hi = np.full(3, -25.0), np.full(3, 25.0)
    m = po.Mesh64(tri)
    mism = 0
    for i in range(3000):
        if i % 3 == 0:
            j = int(rng.integers(tri.shape[0]))
            p = rng.dirichlet([1, 1, 1]) @ tri[j].reshape(3, 3).astype(np.float64)
            ref = j
        else:
            p, ref = rng.uniform(lo, hi), -1
        v = rng.normal(size=3)
        v /= np.linalg.norm(v)
        bound = (10000.0, rng.exponential(5.0), rng.exponential(0.3))[i % 3]
        if m.query(p, v, ref, bound) != m.brute(p, v, ref, bound):
            mism += 1
    assert mism == 0


@pytest.mark.parametrize("case", ["slab", "abdomen"])
def test_common_random_numbers_follow_the_fp32_oracle(oracle_lib, case):
    w = workloads.plain_slab() if case == "slab" else workloads.curved_abdomen(freq=6)
    n = 2000 if case == "slab" else 600
    c = to_case(w)
    r32 = po.run(c, n, rng_mode=po.RNG_PHILOX, seed=1234, exit_records=True, compat=w.compat)
    r64 = po.run64(c, n, seed=1234, exit_records=True, compat=w.compat)
    close = np.all(np.isclose(r32.exit_rec, r64.exit_rec, rtol=1e-3, atol=1e-3), axis=1).mean()
    # thousands of FP32 roundings per photon separate the two; the photons whose trajectories
    # part after a rounding flips a decision are the rest
    assert close > (0.8 if case == "slab" else 0.7), close
    # event counts: the parted photons make independent, heavy-tailed contributions
    tol = 0.03 if case == "slab" else 0.12
    for k in ("scatter", "boundary"):
        assert abs(r32.counters[k] - r64.counters[k]) <= tol * r32.counters[k], k


def test_independent_streams_agree_statistically(oracle_lib):
    w = workloads.plain_slab()
    c = to_case(w)
    a, b = [], []
    for i in range(8):
        r32 = po.run(c, 1500, first=i * 1500, rng_mode=po.RNG_PHILOX, seed=11, compat=w.compat)
        r64 = po.run64(c, 1500, first=i * 1500, seed=12, compat=w.compat)
        a.append(fx.scalars(dict(sft=r32.sft, region=r32.region), 1500))
        b.append(fx.scalars(dict(sft=r64.sft, region=r64.region), 1500))
    z = z_scores(a, b)
    assert np.all(np.abs(z[np.isfinite(z)]) < 3), z


def test_fresnel_in_double_matches_float(oracle_lib):
    L = po.lib()
    for n1, n2 in ((1.0, 1.4), (1.4, 1.0), (1.33, 1.44)):
        for c in (1.0, 0.9, 0.5, 0.2, -0.7):
            a = L.lpo_fresnel(n1, n2, c)
            b = L.lpo64_fresnel(n1, n2, c)
            # a negative cosine (the reference's signed form) cancels in sin(i + t): r >> 1
            # there and only its relative value is meaningful
            assert abs(a - b) <= (2e-6 if c > 0 else 1e-4) * max(1.0, abs(b)), (n1, n2, c, a, b)


@pytest.mark.parametrize("name", sorted(fx.SPEC))
def test_statistics_fixtures_match_the_workloads(name):
    """A fixture is only valid for the exact workload it was made from."""
    path = os.path.join(os.path.dirname(fx.__file__), f"oracle64_{name}.npz")
    if not os.path.isfile(path):
        pytest.skip(f"{path} not generated")
    z = np.load(path)
    assert str(z["mesh_hash"]) == fx.mesh_hash(fx.workload(name))
    assert int(z["B"]) == fx.SPEC[name]["B"] and int(z["n"]) == fx.SPEC[name]["n"]
    assert z["scalars_b"].shape[0] == int(z["B"])
