"""FP64-oracle statistics fixtures: the definitions shared by their maker and their readers.

A fixture holds, for one workload, the batch statistics of an FP64 oracle run
(oracle/lp_oracle64.c): B batches of n photons each, every tally normalised to weight
per launched photon.  For each tally the fixture keeps S1 = sum over batches of the
batch value and S2 = sum of its squares, so a reader gets the mean (S1 / B) and the
variance of the mean ((S2 - S1^2 / B) / (B - 1) / B) of every bin.  Images are stored
at the resolution `SPEC[workload]` names (block sums of the full tally layout), the
voxel grid additionally as its full-resolution mean with the summed variance of the
mean, which is what a relative-L2 comparison needs.

    python tests/golden/fixture64.py [plain_slab|abdomen660|abdomen940 ...]

writes tests/golden/oracle64_<name>.npz (deterministic: fixed seeds and photon ids).
"""
from __future__ import annotations

import hashlib
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
FIX = 2.0 ** 32

# workload name -> (constructor kwargs, photons per batch, batches, seed, image blocks)
#   blocks: per image the block shape of the stored resolution ([y, x, comp] for sft,
#   [alpha, r, comp] for rtd, [z, r, comp] for rz, [z, y, x] for vox); "vox_l2" is the
#   resolution of the voxel relative-L2 comparison.
SPEC = {
    "plain_slab": dict(workload=("plain_slab", {}), n=500_000, B=20, seed=0x64_0011,
                       blocks={"sft": (1, 1, 1), "rtd": (1, 1, 1), "rz": (1, 1, 1), "vox": (3, 5, 5),
                               "vox_l2": (1, 1, 1)}),
    "abdomen660": dict(workload=("curved_abdomen", {"wavelength": 660, "freq": 12}), n=200_000, B=40,
                       seed=0x64_0660,
                       blocks={"sft": (4, 4, 1), "rtd": (2, 4, 1), "rz": (4, 4, 1), "vox": (10, 10, 10),
                               "vox_l2": (5, 5, 5)}),
    "abdomen940": dict(workload=("curved_abdomen", {"wavelength": 940, "freq": 12}), n=200_000, B=20,
                       seed=0x64_0940,
                       blocks={"sft": (4, 4, 1), "rtd": (2, 4, 1), "rz": (4, 4, 1), "vox": (10, 10, 10),
                               "vox_l2": (5, 5, 5)}),
}


def workload(name):
    sys.path.insert(0, ROOT)
    from lightpropagation_b200 import workloads
    fn, kw = SPEC[name]["workload"]
    return getattr(workloads, fn)(**kw)


def mesh_hash(w) -> str:
    """Digest of every input that shapes the statistics, so a fixture refuses a drifted workload."""
    h = hashlib.sha256()
    for a in (w.tri, w.nrm, w.med, w.nmuasg, w.p_start, w.v_start, w.ep0xyz, w.dimensions, w.det_grid):
        h.update(np.ascontiguousarray(a).tobytes())
    h.update(repr((w.fetal_id, w.chance, w.w_threshold, w.factor, tuple(w.vox_n), tuple(w.vox_d), w.n_rbins,
                   w.rbin_dr, None if w.det_r is None else w.det_r.tolist(), w.fiber_radius, w.fiber_na,
                   w.compat)).encode())
    return h.hexdigest()[:32]


def block_sum(a, blocks):
    """Sum of `a` over blocks of the given shape (edges padded with zeros)."""
    a = np.asarray(a, np.float64)
    pad = [(0, (-s) % b) for s, b in zip(a.shape, blocks)]
    a = np.pad(a, pad)
    shp = []
    for s, b in zip(a.shape, blocks):
        shp += [s // b, b]
    return a.reshape(shp).sum(axis=tuple(range(1, 2 * a.ndim, 2)))


def scalars(t, n):
    """R (surface), fetal, T (transmitted) sums and absorption per region (without the
    ambient region 0), per launched photon."""
    sft = np.asarray(t["sft"], np.float64)
    v = [sft[:, :, 0].sum(), sft[:, :, 1].sum(), sft[:, :, 2].sum()] + list(np.asarray(t["region"], np.float64)[1:])
    return np.array(v) / FIX / n


def images(t, n, blocks, vox_shape):
    """Per-photon images at the stored resolutions."""
    out = {}
    for k in ("sft", "rtd", "rz"):
        out[k] = block_sum(np.asarray(t[k], np.float64) / FIX / n, blocks[k])
    vox = np.asarray(t["vox"], np.float64).reshape(vox_shape) / FIX / n
    out["vox"] = block_sum(vox, blocks["vox"])
    out["vox_l2"] = block_sum(vox, blocks["vox_l2"])
    out["rbins"] = np.asarray(t["rbins"], np.float64) / FIX / n
    return out


def stats(s1, s2, B):
    """Mean and variance of the mean from the batch sums."""
    m = s1 / B
    var = np.maximum(s2 - s1 * s1 / B, 0.0) / (B - 1) / B
    return m, var


def make(name):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import pyoracle as po
    from conftest import to_case
    spec = SPEC[name]
    w = workload(name)
    c = to_case(w)
    mesh = po.Mesh64(w.tri)
    n, B, seed, blocks = spec["n"], spec["B"], spec["seed"], spec["blocks"]
    vshape = (w.vox_n[2], w.vox_n[1], w.vox_n[0])
    acc, sc, det, grad, counters = {}, [], [], [], None
    threads = int(os.environ.get("LP_ORACLE_THREADS", "0"))
    t0 = time.time()
    for b in range(B):
        r = po.run64(c, n, first=b * n, seed=seed, compat=w.compat, mesh=mesh, nthreads=threads)
        t = dict(sft=r.sft, rtd=r.rtd, rz=r.rz, vox=r.vox, rbins=r.rbins, region=r.region)
        sc.append(scalars(t, n))
        if r.det.shape[0]:
            det.append(r.det.astype(np.float64) / FIX / n)
            grad.append(r.grad.copy())
        for k, v in images(t, n, blocks, vshape).items():
            if k not in acc:
                acc[k] = [np.zeros_like(v), np.zeros_like(v)]
            acc[k][0] += v
            acc[k][1] += v * v
        cnt = np.array([r.counters[k] for k in po.COUNTER_NAMES], np.float64)
        counters = cnt if counters is None else counters + cnt
        print(f"{name}: batch {b + 1}/{B} done, {time.time() - t0:.0f} s", flush=True)
    out = dict(name=name, workload=w.name, mesh_hash=mesh_hash(w), n=n, B=B, seed=seed,
               scalars_b=np.array(sc), counters=counters, counter_names=np.array(po.COUNTER_NAMES),
               seconds=time.time() - t0)
    for k, (s1, s2) in acc.items():
        if k == "vox_l2":
            m, var = stats(s1, s2, B)
            out["vox_l2_mean"] = m.astype(np.float32)
            out["vox_l2_var_sum"] = np.float64(var.sum())
            continue
        dt = np.float64 if k == "rbins" else np.float32
        out[k + "_s1"] = s1.astype(dt)
        out[k + "_s2"] = s2.astype(dt)
    if det:
        out["det_b"] = np.array(det)
        out["grad_b"] = np.array(grad)
    path = os.path.join(HERE, f"oracle64_{name}.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path} ({os.path.getsize(path) / 1e6:.2f} MB) in {time.time() - t0:.0f} s")


def load(name):
    """The fixture as a dict, with means and variances of the mean of every image."""
    z = np.load(os.path.join(HERE, f"oracle64_{name}.npz"))
    d = {k: z[k] for k in z.files}
    B = int(d["B"])
    for k in ("sft", "rtd", "rz", "vox", "rbins"):
        d[k + "_mean"], d[k + "_var"] = stats(d[k + "_s1"].astype(np.float64), d[k + "_s2"].astype(np.float64), B)
    return d


if __name__ == "__main__":
    for nm in (sys.argv[1:] or list(SPEC)):
        make(nm)
