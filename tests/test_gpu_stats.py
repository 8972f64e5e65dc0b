"""Production CUDA path against the FP64 oracle at high statistics (marked gpu).

The oracle side is a committed fixture (tests/golden/fixture64.py; oracle64_*.npz):
B batches of photons traced by the FP64 oracle (oracle/lp_oracle64.c), reduced to the
sum and sum of squares of every tally's batch values.  Here the production kernel
(fast arithmetic, FP32) traces its own batches of the same workload with another seed,
and the two are compared tally by tally:

  * scalar tallies (surface, fetal and transmitted exit weight, absorption per region,
    ring-detector signals): |z| < 3 each;
  * images (reflectance-by-radius bins, r-z, SFT, RTd, a block-summed voxel grid),
    bin by bin over the bins both sides resolve: max |z| below the Bonferroni bound of
    Student's t for the batch counts, and the mean z^2 near its expectation;
  * the voxel absorption ("fluence") grid at the stated resolution: relative L2
    difference below 1%, with the part the two runs' noise explains reported beside it;
  * derivatives of every ring signal by every region's mua and mus (perturbation Monte
    Carlo): |z| within the Bonferroni bound of Student's t.

z = (mean_gpu - mean_oracle) / sqrt(se_gpu^2 + se_oracle^2), each se from its batches.
GPU results are deterministic for a seed, so each test gives the same outcome every run.
"""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import fixture64 as fx  # noqa: E402
from lightpropagation_b200 import Simulation  # noqa: E402

pytestmark = pytest.mark.gpu

FIX = 2.0 ** 32


def t_bound(n_tests, dof, alpha=1e-3):
    """Two-sided Student-t quantile at the Bonferroni level alpha / n_tests."""
    from scipy import stats
    return float(stats.t.ppf(1.0 - alpha / (2.0 * max(n_tests, 1)), dof))


def gpu_batches(w, spec, n, B, seed, grad=False):
    """B launches of n photons of w (disjoint photon ranges) with the production kernel:
    batch sums S1, S2 of every image at the fixture's resolutions, per-batch scalars,
    rings and derivatives."""
    vshape = (w.vox_n[2], w.vox_n[1], w.vox_n[0])
    acc, sc, det, dmua, dmus = {}, [], [], [], []
    with Simulation(0) as s:
        w.apply(s, seed=seed)
        s.set_arithmetic(False)
        if grad:
            s.set_gradient(True)
        for b in range(B):
            s.zero()
            s.run(n, 10 ** 11 + b * n)
            t = s.tallies()
            sc.append(fx.scalars(t, n))
            if t["det"].shape[0]:
                det.append(t["det"].astype(np.float64) / FIX / n)
            if grad:
                g = s.gradient()
                dmua.append(g["d_mua"])
                dmus.append(g["d_mus"])
            for k, v in fx.images(t, n, spec["blocks"], vshape).items():
                if k not in acc:
                    acc[k] = [np.zeros_like(v), np.zeros_like(v)]
                acc[k][0] += v
                acc[k][1] += v * v
    out = {"scalars_b": np.array(sc), "B": B}
    for k, (s1, s2) in acc.items():
        out[k + "_mean"], out[k + "_var"] = fx.stats(s1, s2, B)
    if det:
        out["det_b"] = np.array(det)
    if grad:
        out["dmua_b"], out["dmus_b"] = np.array(dmua), np.array(dmus)
    return out


def batch_z(a, b):
    """z of the difference of the means of two batch samples [B, ...]."""
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    se2 = a.var(0, ddof=1) / a.shape[0] + b.var(0, ddof=1) / b.shape[0]
    with np.errstate(divide="ignore", invalid="ignore"):
        return np.where(se2 > 0, (a.mean(0) - b.mean(0)) / np.sqrt(se2), 0.0)


def image_z(g, o, key, min_rel_se=0.1):
    """Per-bin z over the bins that both sides resolve (relative standard error of the
    mean below min_rel_se on each side).  A bin fed by a handful of heavy photons (the
    transmitted and fetal components far from the source) has a skewed batch
    distribution whose sample variance understates the error of its mean; 10 % keeps
    those out."""
    mg, vg, mo, vo = g[key + "_mean"], g[key + "_var"], o[key + "_mean"], o[key + "_var"]
    ok = (mo > 0) & (mg > 0) & (vo > 0) & (vg > 0)
    ok &= (np.sqrt(vo) < min_rel_se * mo) & (np.sqrt(vg) < min_rel_se * mg)
    z = (mg[ok] - mo[ok]) / np.sqrt(vg[ok] + vo[ok])
    return z


def oracle_derivatives(o, w):
    """Per-batch ring-signal derivatives from the oracle's perturbation-MC sums."""
    g = o["grad_b"]                              # [B, D, R, 5]
    n = float(o["n"])
    mus = np.asarray(w.nmuasg, np.float64)[:, 2]
    f = float(w.factor)
    dmua = -g[..., 0] / f / n
    with np.errstate(divide="ignore", invalid="ignore"):
        dmus = np.where(mus > 0, (g[..., 1] / mus - g[..., 0] / f) / n, 0.0)
    return dmua, dmus


def check_images(g, o, keys, dof):
    report = {}
    for k in keys:
        z = image_z(g, o, k)
        assert z.size > 10, (k, z.size)
        bound = t_bound(z.size, dof)
        report[k] = (z.size, float(np.abs(z).max()), float(np.mean(z * z)))
        print(f"{k}: {z.size} bins, max |z| {report[k][1]:.2f} (bound {bound:.2f}), mean z^2 {report[k][2]:.3f}")
        assert np.abs(z).max() < bound, f"{k}: max |z| {np.abs(z).max():.2f} >= {bound:.2f} over {z.size} bins"
        # E[t^2] = dof / (dof - 2) for Student's t; allow for the correlation of bins
        assert np.mean(z * z) < 1.5 * dof / (dof - 2), f"{k}: mean z^2 {np.mean(z * z):.3f}"
    return report


def voxel_l2(g, o):
    """Relative L2 difference of the voxel grids at the L2 resolution, and the part of it
    that the statistical noise of the two runs explains."""
    mg, mo = g["vox_l2_mean"], o["vox_l2_mean"].astype(np.float64)
    nrm = np.linalg.norm(mo)
    rel = np.linalg.norm(mg - mo) / nrm
    noise = np.sqrt(g["vox_l2_var"].sum() + float(o["vox_l2_var_sum"])) / nrm
    return float(rel), float(noise)


@pytest.fixture(scope="module")
def slab_pair():
    o = fx.load("plain_slab")
    w = fx.workload("plain_slab")
    assert fx.mesh_hash(w) == str(o["mesh_hash"]), "the workload changed since the fixture was made"
    g = gpu_batches(w, fx.SPEC["plain_slab"], 5_000_000, 20, seed=0x5EED)
    return g, o, w


def test_slab_scalar_tallies_vs_fp64_oracle(slab_pair):
    """1e8 production photons on the 3-layer slab against 1e7 FP64-oracle photons:
    surface, fetal and transmitted weight and absorption per region, |z| < 3 each."""
    g, o, _ = slab_pair
    z = batch_z(g["scalars_b"], o["scalars_b"])
    print("slab scalar z:", np.round(z, 2))
    assert np.all(np.abs(z) < 3), z


def test_slab_images_vs_fp64_oracle(slab_pair):
    g, o, _ = slab_pair
    dof = min(g["B"], int(o["B"])) - 1
    check_images(g, o, ("rbins", "rz", "sft", "rtd", "vox"), dof)


def test_slab_voxel_fluence_relative_l2(slab_pair):
    """The accuracy bar: relative L2 of the 1 mm voxel absorption grid below 1% at 1e8
    photons; the noise of the two runs explains most of what remains."""
    g, o, _ = slab_pair
    rel, noise = voxel_l2(g, o)
    print(f"slab voxel relative L2 {rel:.4f}, noise of the two runs {noise:.4f}")
    assert rel < 0.01, (rel, noise)
    assert rel * rel - noise * noise < 0.005 ** 2, f"relative L2 {rel:.4f}, noise alone {noise:.4f}"


@pytest.fixture(scope="module", params=["abdomen660", "abdomen940"])
def abdomen_pair(request):
    name = request.param
    o = fx.load(name)
    w = fx.workload(name)
    assert fx.mesh_hash(w) == str(o["mesh_hash"]), "the workload changed since the fixture was made"
    g = gpu_batches(w, fx.SPEC[name], 2_000_000, 20, seed=0x5EED + 1, grad=True)
    return g, o, w


def test_abdomen_scalar_tallies_and_rings_vs_fp64_oracle(abdomen_pair):
    """Curved abdomen (14,400 triangles, fibre source, corrected physics): 4e7 production
    photons against 4e6 FP64-oracle photons, |z| < 3 per scalar tally and per ring."""
    g, o, _ = abdomen_pair
    z = batch_z(g["scalars_b"], o["scalars_b"])
    zr = batch_z(g["det_b"][:, :, 0], o["det_b"][:, :, 0])
    print(f"{o['name']} scalar z:", np.round(z, 2), "ring z:", np.round(zr, 2))
    assert np.all(np.abs(z) < 3), z
    assert np.all(np.abs(zr) < 3), zr


def test_abdomen_images_vs_fp64_oracle(abdomen_pair):
    g, o, _ = abdomen_pair
    dof = min(g["B"], int(o["B"])) - 1
    check_images(g, o, ("rbins", "rz", "sft", "rtd", "vox"), dof)


def test_abdomen_voxel_fluence_relative_l2(abdomen_pair):
    g, o, _ = abdomen_pair
    rel, noise = voxel_l2(g, o)
    print(f"{o['name']} voxel relative L2 {rel:.4f}, noise of the two runs {noise:.4f}")
    assert rel < 0.01, (rel, noise)


def test_abdomen_derivatives_vs_fp64_perturbation_mc(abdomen_pair):
    """dS_d/dmua_r and dS_d/dmus_r of the 6 rings x 5 tissue regions (60 per wavelength,
    120 over both) from the adjoint sums of the production kernel against the FP64
    oracle's perturbation-MC sums."""
    g, o, w = abdomen_pair
    oa, os_ = oracle_derivatives(o, w)
    za = batch_z(g["dmua_b"][:, :, 1:], oa[:, :, 1:])
    zs = batch_z(g["dmus_b"][:, :, 1:], os_[:, :, 1:])
    z = np.concatenate([za.ravel(), zs.ravel()])
    print(f"{o['name']} derivatives: max |z| {np.abs(z).max():.2f} over {z.size}")
    assert z.size == 60
    bound = t_bound(z.size, min(g["B"], int(o["B"])) - 1, alpha=1e-2)
    assert np.abs(z).max() < bound, (np.abs(z).max(), bound)
