"""Inverse loop: Gauss-Newton recovery of fetal SpO2 and fetal blood fraction from the
ring-detector signals at 660 and 940 nm, with batched forward + gradient launches.

Ground truths: `truths` seeded (fetal SpO2 U(30, 70) %, fetal blood fraction U(2, 8) %)
on the large deformed abdomen (placenta, 3-octave noise displacement); maternal SpO2 and
blood fraction are known.  Their synthetic signals come from one batch of
2 x truths instances (both wavelengths) at `truth_photons` each.  The fit starts every
truth at (50 %, 5 %) and takes `iterations` damped Gauss-Newton steps on the fetal-head
absorption at each wavelength; each step is ONE batched launch of all 2 x truths
instances at `fit_photons` each with the adjoint sums on, giving the signals and
d(signal)/d(mua) of the fetal head.  Since mua = background + blood fraction x blood
absorption(SpO2) is linear in (bf, bf SpO2), the two fitted absorptions give SpO2 and the
blood fraction by a 2x2 solve.  Each step traces fresh photons and the estimate is the
mean of the second half of the iterates (common random numbers do not make this
objective smooth: a change of the head's absorption moves roulette decisions and, through
mua + mus, the step lengths inside the head, so a detected photon's weight jumps).  A
step changes an absorption by at most `max_step` of its value (trust region), which
keeps a noisy derivative from throwing the fit out of range.

The fetal head lies 40 mm deep under 20-27 mm of maternal tissue: few detected photons
reach it, so the recovered SpO2 error is set by the photon budget (see the report).

    python -m lightpropagation_b200.inverse [--truths 64] [--truth-photons 1e7]
        [--fit-photons 1e6] [--iterations 10] [--freq 129] [--json out.json]

No reference counterpart: the reference has no inverse solver.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import workloads as W
from .batch import Batch, Instance
from .propagation import Simulation

FETAL = 5
WAVELENGTHS = (660, 940)
MATERNAL_SPO2, MATERNAL_BF = 0.97, 0.05


def table(wavelength: int, spo2_f: float, bf_f: float) -> np.ndarray:
    """(n, mua, mus, g) of the 7 regions of the deformed abdomen."""
    t = W.tissue_table(wavelength, MATERNAL_SPO2, spo2_f, MATERNAL_BF, bf_f)
    return np.vstack([t, np.array(W.PLACENTA, np.float32)]).astype(np.float32)


def mua_head(wavelength: int, spo2_f: float, bf_f: float) -> float:
    """Absorption of the fetal head [1/mm] (background + blood share x fraction x blood)."""
    return float(W.BACKGROUND_MUA[wavelength][FETAL] + W.BLOOD_SHARE[FETAL] * bf_f * W.blood_mua(spo2_f, wavelength))


def saturation_of(mua_pair) -> np.ndarray:
    """(SpO2, blood fraction) from the fetal-head absorption at 660 and 940 nm: with
    a = (mua - background) / (share ln10 C / 10) = bf e_de + bf SpO2 (e_ox - e_de) at each
    wavelength, (bf, bf SpO2) solve a 2x2 linear system."""
    A, rhs = [], []
    scale = W.BLOOD_SHARE[FETAL] * np.log(10.0) * W.HB_MOLAR / 10.0
    for k, wl in enumerate(WAVELENGTHS):
        e_ox, e_de = W.HB_EXTINCTION[wl]
        A.append([e_de, e_ox - e_de])
        rhs.append((mua_pair[k] - W.BACKGROUND_MUA[wl][FETAL]) / scale)
    bf, bfs = np.linalg.solve(np.array(A), np.array(rhs))
    bf = max(bf, 1e-6)
    return np.array([float(np.clip(bfs / bf, 0.0, 1.0)), float(bf)])


def instances(theta, n, first0, mua=None):
    """Two instances (660, 940 nm) per row of theta (SpO2, blood fraction); the fetal
    head's mua is taken from `mua` ([rows, 2]) when given."""
    out = []
    for i, (s, b) in enumerate(theta):
        for k, wl in enumerate(WAVELENGTHS):
            t = table(wl, s, b)
            if mua is not None:
                t[FETAL, 1] = np.float32(mua[i, k])
            out.append(Instance(context=0, nmuasg=t, n_photons=int(n), first=int(first0 + (2 * i + k) * n)))
    return out


def gn_step(signal, se, dsd, s_obs, e_obs, lam=0.1):
    """One damped Gauss-Newton step on a scalar absorption from the signals of the rings
    that saw light: relative residuals, weights from both relative errors."""
    ok = (s_obs > 0) & np.isfinite(e_obs) & (signal > 0)
    if not ok.any():
        return 0.0
    jac = dsd[ok] / s_obs[ok]
    r = (signal[ok] - s_obs[ok]) / s_obs[ok]
    wt = 1.0 / np.maximum(np.hypot(se[ok] / signal[ok], e_obs[ok]), 1e-6) ** 2
    a = float(np.sum(wt * jac * jac))
    if a <= 0.0:
        return 0.0
    return -float(np.sum(wt * jac * r)) / (a * (1.0 + lam))


def fit(truths: int = 64, truth_photons: float = 1e7, fit_photons: float = 1e6, iterations: int = 10,
        freq: int = 129, seed: int = 6, rings=(1, 2, 3, 4, 5), device: int = 0, log=print,
        truth_first: int = 10 ** 13, max_step: float = 0.3, crn: bool = False) -> dict:
    """Run the fit.  truth_first is the first photon id of the observations (disjoint from
    the fit's photons by default).  Each step traces fresh photons unless crn is set, and
    the reported estimate averages the absorptions of the second half of the steps, which
    damps the Monte Carlo noise of the single steps."""
    t_setup = time.perf_counter()
    w = W.deformed_abdomen(freq=freq)
    sim = w.apply(Simulation(device), seed=0x4C50)
    rng = np.random.default_rng(seed)
    truth = np.stack([rng.uniform(0.30, 0.70, truths), rng.uniform(0.02, 0.08, truths)], 1)
    truth_mua = np.array([[mua_head(wl, *t) for wl in WAVELENGTHS] for t in truth])
    b = Batch([sim])
    rings = list(rings)
    setup_s = time.perf_counter() - t_setup

    t0 = time.perf_counter()
    b.set_instances(instances(truth, truth_photons, truth_first))
    b.run()
    s_obs, e_obs = b.ring_signals()
    s_obs = s_obs.reshape(truths, 2, -1)[:, :, rings]
    e_obs = e_obs.reshape(truths, 2, -1)[:, :, rings]
    truth_s = time.perf_counter() - t0
    log(f"observations: {2 * truths} instances x {truth_photons:.0e} photons in {truth_s:.1f} s")

    mua = np.array([[mua_head(wl, 0.5, 0.05) for wl in WAVELENGTHS]] * truths)
    theta = np.array([saturation_of(m) for m in mua])
    b.set_gradient(True)
    history = []
    t0 = time.perf_counter()
    launch_ms = 0.0
    tail = []                       # iterates of the second half, averaged at the end
    for it in range(iterations):
        first0 = 0 if crn else it * 2 * truths * int(fit_photons)
        b.set_instances(instances(theta, fit_photons, first0, mua))
        b.run()
        launch_ms += b.last_ms()
        for i in range(truths):
            for k, wl in enumerate(WAVELENGTHS):
                g = b.gradient(2 * i + k)
                step = gn_step(g["signal"][rings], g["signal_se"][rings], g["d_mua"][rings, FETAL],
                               s_obs[i, k], e_obs[i, k])
                step = float(np.clip(step, -max_step * mua[i, k], max_step * mua[i, k]))
                mua[i, k] = max(mua[i, k] + step, W.BACKGROUND_MUA[wl][FETAL] + 1e-5)
        if it >= iterations // 2:
            tail.append(mua.copy())
        est = np.mean(tail, axis=0) if tail else mua
        theta = np.array([saturation_of(m) for m in est])
        err = np.abs(theta[:, 0] - truth[:, 0])
        history.append({"iteration": it + 1, "mean_abs_spo2_error": float(err.mean()),
                        "max_abs_spo2_error": float(err.max()),
                        "mean_abs_bf_error": float(np.abs(theta[:, 1] - truth[:, 1]).mean()),
                        "mean_rel_mua_error": [float(x) for x in np.abs(est / truth_mua - 1).mean(0)]})
        log(f"iteration {it + 1}: mean |SpO2 error| {100 * err.mean():.2f} points, max {100 * err.max():.2f}; "
            f"mean relative mua error {np.abs(est / truth_mua - 1).mean(0)}")
    fit_s = time.perf_counter() - t0
    err = theta[:, 0] - truth[:, 0]
    out = {"workload": w.name, "triangles": int(w.n_tri), "truths": truths,
           "truth_photons_per_instance": truth_photons, "fit_photons_per_instance": fit_photons,
           "iterations": iterations, "rings_used_mm": [float(x) for x in np.array(W.RING_SEPARATIONS_MM)[rings]],
           "spo2_error_points": {"mean_abs": float(100 * np.abs(err).mean()),
                                 "rms": float(100 * np.sqrt((err ** 2).mean())),
                                 "max_abs": float(100 * np.abs(err).max())},
           "bf_error_mean_abs": float(np.abs(theta[:, 1] - truth[:, 1]).mean()),
           "mua_rel_error_mean": [float(x) for x in np.abs(est / truth_mua - 1).mean(0)],
           "time_to_fit_s": fit_s, "fit_device_s": launch_ms * 1e-3, "observation_s": truth_s,
           "setup_s": setup_s, "history": history}
    b.close()
    sim.close()
    return out


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--truths", type=int, default=64)
    ap.add_argument("--truth-photons", type=float, default=1e7)
    ap.add_argument("--fit-photons", type=float, default=1e6)
    ap.add_argument("--iterations", type=int, default=10)
    ap.add_argument("--freq", type=int, default=129)
    ap.add_argument("--seed", type=int, default=6)
    ap.add_argument("--json", default="")
    a = ap.parse_args()
    out = fit(a.truths, a.truth_photons, a.fit_photons, a.iterations, a.freq, a.seed)
    print(json.dumps({k: v for k, v in out.items() if k != "history"}))
    if a.json:
        with open(a.json, "w") as f:
            json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
