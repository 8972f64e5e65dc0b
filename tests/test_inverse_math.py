"""CPU checks of the inverse loop's algebra (lightpropagation_b200.inverse): the
two-wavelength absorption -> (SpO2, blood fraction) solve inverts the forward mixing
model, and the damped Gauss-Newton step on a scalar absorption reaches the minimum of an
exponential signal model in a few steps.  The GPU test runs the loop itself."""
import numpy as np

from lightpropagation_b200 import inverse as I
from lightpropagation_b200 import meshes


def test_saturation_inverts_mixing_model():
    for s, b in [(0.3, 0.02), (0.5, 0.05), (0.7, 0.08), (0.95, 0.03)]:
        m = [I.mua_head(wl, s, b) for wl in I.WAVELENGTHS]
        got = I.saturation_of(m)
        assert abs(got[0] - s) < 1e-9 and abs(got[1] - b) < 1e-12


def test_gauss_newton_step_converges_on_exponential_model():
    L = np.array([2.0, 5.0, 9.0, 14.0])           # mean path length in the region per ring (mm)
    s0 = np.array([1e-3, 1e-4, 1e-5, 1e-6])
    true_mu = 0.04

    def model(mu):
        return s0 * np.exp(-L * (mu - true_mu))

    obs = model(true_mu)
    mu = 0.06
    for _ in range(6):
        s = model(mu)
        step = I.gn_step(s, 0.01 * s, -L * s, obs, np.full(4, 0.01), lam=0.0)
        mu += step
    assert abs(mu - true_mu) < 1e-6


def test_deformed_mesh_generator_counts_and_regions():
    tri, nrm, med, pole = meshes.deformed_abdomen(freq=10)
    assert tri.shape == (6 * 2000, 9)
    assert set(map(tuple, np.unique(med, axis=0))) == {(1, 0), (2, 1), (3, 2), (4, 3), (5, 4), (6, 4)}
    assert abs(pole[2] + 100.0) <= 3.0
    n = meshes.octave_noise(np.random.default_rng(0).uniform(-100, 100, (20000, 3)), 5)
    assert np.all(np.abs(n) <= 1.0) and 0.05 < n.std() < 0.6
    # a fixed field: one point gives the same value alone and among others
    p = np.array([[10.0, -20.0, 30.0]])
    assert meshes.octave_noise(p, 5)[0] == meshes.octave_noise(np.vstack([p, p * 2]), 5)[0]
