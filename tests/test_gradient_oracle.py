"""The perturbation-Monte-Carlo gradient of the oracle against its own central finite
differences with common random numbers (CPU only).

The oracle keeps, per photon, the path length L_r and interaction count k_r in every
region and adds s * L_r and s * k_r to FP64 sums when the photon scores weight s in a
ring detector; dS/dmua_r = -sum s L_r / N and dS/dmus_r = (sum s k_r / mus_r - sum s L_r) / N.
The finite difference perturbs one coefficient by +-1% and reruns the same photon ids
(same Philox streams).  Both estimate the same derivative with different noise, so the
test compares them batch by batch: the mean of the per-batch differences must be within
4 standard errors of zero, and for the dominant derivatives within 5% of their value.
This pins the estimator the CUDA kernel implements (the GPU tests compare the kernel
with the oracle)."""
import numpy as np

from conftest import po, to_case
from lightpropagation_b200 import workloads

RINGS = np.array([[0.5, 1.5], [1.5, 3.0], [3.0, 6.0], [6.0, 10.0]], np.float32)


def _slab():
    w = workloads.plain_slab()
    w.compat = 0          # corrected physics: light reaches every layer
    w.det_r = RINGS
    return w


def _signal(case, n, first, compat):
    r = po.run(case, n, first=first, seed=5, compat=compat, nthreads=0)
    return r, r.det[:, 0].astype(np.float64) / 2.0 ** 32 / n


def test_pmc_gradient_matches_central_differences(oracle_lib):
    w = _slab()
    base = np.array(w.nmuasg, np.float32)
    params = [(1, 1), (2, 1), (1, 2)]      # (region, column): mua skin, mua fat, mus skin
    B, n = 6, 8000
    diffs = {p: [] for p in params}
    pmc_all = {p: [] for p in params}
    for b in range(B):
        case = to_case(w)
        r0, _ = _signal(case, n, b * n, w.compat)
        _, d_mua, d_mus = po.gradient(r0, case, n)
        for reg, col in params:
            h = np.float32(0.01) * base[reg, col]
            s = []
            for sgn in (1, -1):
                m = base.copy()
                m[reg, col] = base[reg, col] + sgn * h
                c2 = to_case(w)
                c2.nmuasg = m
                s.append(_signal(c2, n, b * n, w.compat)[1])
            fd = (s[0] - s[1]) / (np.float64(base[reg, col] + h) - np.float64(base[reg, col] - h))
            pmc = (d_mua if col == 1 else d_mus)[:, reg]
            diffs[(reg, col)].append(pmc - fd)
            pmc_all[(reg, col)].append(pmc)
    for p in params:
        d = np.array(diffs[p])
        m = d.mean(0)
        se = d.std(0, ddof=1) / np.sqrt(B)
        z = np.abs(m) / np.maximum(se, 1e-12)
        assert np.all(z < 4.0), (p, m, se)
        g = np.array(pmc_all[p]).mean(0)
        if p[1] == 1:   # absorption derivatives are large and well resolved
            assert np.all(np.abs(m) <= 0.05 * np.abs(g) + 4 * se), (p, m, g)


def test_gradient_sums_are_zero_without_rings(oracle_lib):
    w = workloads.plain_slab()
    r = po.run(to_case(w), 200, seed=5, compat=w.compat, nthreads=1)
    assert r.grad.shape[0] == 0 and r.det.shape[0] == 0
