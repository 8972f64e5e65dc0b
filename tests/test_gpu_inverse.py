"""Inverse loop on the GPU, small: a coarse deformed abdomen, two truths, four Gauss-
Newton steps, each one batched forward + gradient launch of all instances.  Checks that
the loop runs end to end and keeps its estimates physical; the accuracy of the recovered
SpO2 is a matter of photon budget and is reported by the full run, not asserted here."""
import numpy as np
import pytest

from lightpropagation_b200 import inverse

pytestmark = pytest.mark.gpu


def test_inverse_loop_runs_on_batched_gradients():
    out = inverse.fit(truths=2, truth_photons=400_000, fit_photons=200_000, iterations=4, freq=16, seed=1,
                      log=lambda *a: None)
    assert out["triangles"] == 6 * 20 * 16 * 16
    assert len(out["history"]) == 4
    for h in out["history"]:
        assert np.isfinite(h["mean_abs_spo2_error"]) and 0.0 <= h["mean_abs_spo2_error"] <= 1.0
        assert all(np.isfinite(h["mean_rel_mua_error"]))
    assert out["time_to_fit_s"] > 0 and out["fit_device_s"] > 0
