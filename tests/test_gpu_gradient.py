"""Differentiation on the GPU: the adjoint path-length / interaction-count sums of the
transport kernel against the oracle's perturbation-MC sums (same photons, reference
arithmetic), against central finite differences with common random numbers (production
arithmetic, high statistics), and through the forward/backward API.

Tolerances: each derivative agrees with its finite difference within the Bonferroni
bound of Student's t at the precision its batches give (see the test); sums over the same photons in reference arithmetic agree
with the oracle within 4 standard errors (only photons whose float trajectories part
contribute to the difference); transport tallies are bit-identical with differentiation
on and off."""
import numpy as np
import pytest

from conftest import po, to_case
from lightpropagation_b200 import Simulation, workloads

pytestmark = pytest.mark.gpu

RINGS = np.array([[0.5, 1.5], [1.5, 3.0], [3.0, 6.0], [6.0, 10.0]], np.float32)
KEYS = ("sft", "rtd", "rz", "vox", "rbins", "region", "det")


def _slab():
    w = workloads.plain_slab()
    w.compat = 0
    w.det_r = RINGS
    return w


def _run(w, nm, n, seed, grad, exact=False, first=0):
    with Simulation(0) as s:
        w.apply(s, seed=seed)
        s.set_media(nm)
        s.set_arithmetic(exact)
        s.set_gradient(grad)
        s.zero()
        s.run(n, first)
        return s.tallies(), (s.gradient() if grad else None), s.kernel_ms()


def test_differentiation_leaves_transport_unchanged():
    w = _slab()
    nm = np.array(w.nmuasg, np.float32)
    a, _, _ = _run(w, nm, 50000, 3, False)
    b, g, _ = _run(w, nm, 50000, 3, True)
    for k in KEYS:
        assert np.array_equal(a[k], b[k]), k
    assert g["n_photons"] == 50000
    assert np.allclose(g["signal"], b["det"][:, 0] / 2.0 ** 32 / 50000)


@pytest.mark.parametrize("case", ["slab", "abdomen"])
def test_gradient_sums_match_oracle(oracle_lib, case):
    if case == "slab":
        w, n = _slab(), 20000
    else:
        w, n = workloads.curved_abdomen(freq=12), 1500
    nm = np.array(w.nmuasg, np.float32)
    _, g, _ = _run(w, nm, n, 5, True, exact=True)
    c = to_case(w)
    r = po.run(c, n, seed=5, compat=w.compat, nthreads=0)
    S, d_mua, d_mus = po.gradient(r, c, n)
    # oracle standard errors from its second moments (same formulas as lp_get_gradient)
    G = r.grad
    mus = np.asarray(c.nmuasg, np.float64)[:, 2]

    def se(sx, sxx):
        return np.sqrt(np.maximum(sxx / n - (sx / n) ** 2, 0.0) / n)

    se_a = se(-G[:, :, 0], G[:, :, 2])
    with np.errstate(divide="ignore", invalid="ignore"):
        se_s = np.where(mus > 0, se(G[:, :, 1] / mus - G[:, :, 0],
                                    G[:, :, 3] / mus ** 2 + G[:, :, 2] - 2 * G[:, :, 4] / mus), 0.0)
    # rings with enough detections for a statistical comparison (relative error < 20 %)
    rows = g["signal_se"] < 0.2 * np.maximum(g["signal"], 1e-300)
    assert rows.sum() >= 2
    tol_sig = 4 * np.hypot(g["signal_se"], se(S * n, r.det[:, 1] / 2.0 ** 32))
    assert np.all(np.abs(g["signal"] - S)[rows] <= tol_sig[rows]), (g["signal"], S)
    for key, ora, s_ora in (("d_mua", d_mua, se_a), ("d_mus", d_mus, se_s)):
        tol = 4 * np.hypot(g[key + "_se"], s_ora) + 1e-12
        bad = (np.abs(g[key] - ora) > tol) & rows[:, None]
        assert not bad.any(), (key, np.argwhere(bad), g[key][bad], ora[bad], tol[bad])


def test_adjoint_matches_central_differences_all_120():
    """All 120 derivatives of the ring signals (5 tissue regions x 6 rings x (mua, mus) x 2
    wavelengths, on the curved abdomen at 40,000 triangles): the adjoint sums of one
    differentiated pass against central differences (+-5 %, common random numbers: the
    same photon ids at both parameter values), B batches of n photons each
    (LP_FD_PHOTONS, default 4e7 per evaluation).  The batch-to-batch spread of
    (adjoint - difference) gives the standard error se of the comparison.

    A difference of two Monte Carlo runs is noisy even with common random numbers: a
    photon whose trajectory flips (a Fresnel or roulette draw that falls the other way, a
    ring it now misses) adds its whole weight / 2h, so the variance falls only as 1 / h.
    +-5 % keeps the central difference's own error (h^2 / 6 times the third derivative,
    a few 0.1 % here) well below that noise.  Every derivative is compared at the
    precision the batches give: |adjoint - difference| / se below the two-sided
    Student-t quantile (B - 1 degrees of freedom) at the Bonferroni level 1e-2 / 120, so
    that the 120 tests together fail by chance with probability below 1 %; the mean of
    the 120 squared ratios stays near its expectation (a bias shared by many
    derivatives shows there first); and at least 4 derivatives (the strongest: skin, fat
    and uterus mua at the nearest rings) are measured to 3 % or better, so that the
    comparison has teeth where the signal is."""
    import os
    from scipy import stats
    total = int(float(os.environ.get("LP_FD_PHOTONS", "4e7")))
    B = 20
    n = total // B
    seed = 11
    report, bad, z2 = [], [], []
    resolved = compared = 0
    t_max = float(stats.t.ppf(1.0 - 1e-2 / (2 * 120), B - 1))
    for lam in (660, 940):
        w = workloads.curved_abdomen(wavelength=lam, freq=20)
        nm = np.array(w.nmuasg, np.float32)
        params = [(reg, col) for reg in range(1, nm.shape[0]) for col in (1, 2)]
        adj = {p: [] for p in params}
        fdv = {p: [] for p in params}
        with Simulation(0) as s:
            w.apply(s, seed=seed)
            s.set_gradient(True)

            def signal(m, b):
                s.set_media(m)
                return s.forward(n, b * n)

            for b in range(B):
                signal(nm, b)
                g = s.gradient()
                for reg, col in params:
                    h = np.float32(0.05) * nm[reg, col]
                    m_p, m_m = nm.copy(), nm.copy()
                    m_p[reg, col] = nm[reg, col] + h
                    m_m[reg, col] = nm[reg, col] - h
                    fd = (signal(m_p, b) - signal(m_m, b)) / (np.float64(m_p[reg, col]) - np.float64(m_m[reg, col]))
                    adj[(reg, col)].append(g["d_mua" if col == 1 else "d_mus"][:, reg])
                    fdv[(reg, col)].append(fd)
        for p in params:
            a, f = np.array(adj[p]), np.array(fdv[p])
            se = (a - f).std(0, ddof=1) / np.sqrt(B)
            am, fm = a.mean(0), f.mean(0)
            for d in range(am.size):
                compared += 1
                res = se[d] <= 0.03 * abs(fm[d])
                resolved += int(res)
                z = (am[d] - fm[d]) / se[d] if se[d] > 0 else 0.0
                z2.append(z * z)
                report.append((lam, p[0], "mua" if p[1] == 1 else "mus", d, am[d], fm[d], se[d], res))
                if not abs(am[d] - fm[d]) <= t_max * se[d] + 1e-300:
                    bad.append(report[-1])
    for r in report:
        print("%d nm region %d %s ring %d: adjoint %.6g difference %.6g se %.2g %s" %
              (r[0], r[1], r[2], r[3], r[4], r[5], r[6], "resolved" if r[7] else ""))
    mz2 = float(np.mean(z2))
    print(f"{resolved} of {compared} derivatives resolved to 3 % (se); t bound {t_max:.2f}; mean z^2 {mz2:.3f}")
    assert not bad, bad
    assert compared == 120
    # E[t^2] = dof / (dof - 2) = 1.12 for 19 degrees of freedom; the sd of a mean of 120 is ~0.16
    assert mz2 < 2.0, mz2
    assert resolved >= 4, resolved


def test_forward_backward_and_autograd():
    import torch
    from lightpropagation_b200 import diff
    w = _slab()
    nm = np.array(w.nmuasg, np.float32)
    with Simulation(0) as s:
        w.apply(s, seed=21)
        sig = s.forward(200000)
        g = s.gradient()
        up = np.array([1.0, -2.0, 0.5, 3.0])
        gm, gs = s.backward(up)
        assert np.allclose(gm, up @ g["d_mua"]) and np.allclose(gs, up @ g["d_mus"])
        assert np.allclose(sig, g["signal"])
        mua = torch.tensor(nm[:, 1].astype(np.float64), requires_grad=True)
        mus = torch.tensor(nm[:, 2].astype(np.float64), requires_grad=True)
        out = diff.ring_signals(s, nm, mua, mus, 200000)
        (out * torch.from_numpy(up)).sum().backward()
        assert np.allclose(out.detach().numpy(), sig)
        assert np.allclose(mua.grad.numpy(), gm) and np.allclose(mus.grad.numpy(), gs)


def test_gradient_rejects_too_many_regions():
    w = _slab()
    nm = np.tile(np.array(w.nmuasg, np.float32), (3, 1))   # 12 regions
    with Simulation(0) as s:
        w.apply(s, seed=1)
        s.set_media(nm)
        s.set_gradient(True)
        with pytest.raises(Exception, match="at most 8 regions"):
            s.run(100)
