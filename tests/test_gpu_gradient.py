"""Differentiation on the GPU: the adjoint path-length / interaction-count sums of the
transport kernel against the oracle's perturbation-MC sums (same photons, reference
arithmetic), against central finite differences with common random numbers (production
arithmetic, high statistics), and through the forward/backward API.

Tolerances: derivatives agree with finite differences within 2% of their value or 4
standard errors of the adjoint estimate, whichever is larger; sums over the same photons
in reference arithmetic agree with the oracle within 4 standard errors (only photons whose
float trajectories part contribute to the difference); transport tallies are bit-identical
with differentiation on and off."""
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


def test_adjoint_matches_central_differences():
    """4e6 photons in 8 batches; per batch the adjoint derivative and the central
    difference (+-1 %, same photon ids) of every tissue region's mua and mus for every
    ring.  The batch-to-batch spread of (adjoint - difference) gives the standard error
    of the comparison, which includes the finite difference's own noise."""
    w = _slab()
    nm = np.array(w.nmuasg, np.float32)
    B, n, seed = 8, 500_000, 11
    params = [(reg, col) for reg in (1, 2, 3) for col in (1, 2)]
    adj = {p: [] for p in params}
    fdv = {p: [] for p in params}
    for b in range(B):
        with Simulation(0) as s:
            w.apply(s, seed=seed)
            s.set_gradient(True)

            def signal(m):
                s.set_media(m)
                return s.forward(n, b * n)

            signal(nm)
            g = s.gradient()
            for reg, col in params:
                h = np.float32(0.01) * nm[reg, col]
                m_p, m_m = nm.copy(), nm.copy()
                m_p[reg, col] = nm[reg, col] + h
                m_m[reg, col] = nm[reg, col] - h
                fd = (signal(m_p) - signal(m_m)) / (np.float64(m_p[reg, col]) - np.float64(m_m[reg, col]))
                adj[(reg, col)].append(g["d_mua" if col == 1 else "d_mus"][:, reg])
                fdv[(reg, col)].append(fd)
    resolved = 0
    for p in params:
        a, f = np.array(adj[p]), np.array(fdv[p])
        d = a - f
        se = d.std(0, ddof=1) / np.sqrt(B)
        am, fm = a.mean(0), f.mean(0)
        tol = np.maximum(0.02 * np.abs(fm), 4 * se)
        print("region %d %s adjoint %s difference %s se %s" % (p[0], "mua" if p[1] == 1 else "mus",
                                                            np.array2string(am, precision=6),
                                                            np.array2string(fm, precision=6),
                                                            np.array2string(se, precision=2)))
        assert np.all(np.abs(am - fm) <= tol), (p, am, fm, se)
        resolved += int(np.sum(4 * se <= 0.02 * np.abs(fm)))
    assert resolved >= 1      # at least one derivative is resolved to better than 2 % here


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
