"""Batches: many transport instances in one persistent launch (lp_batch_* of the C ABI).

An instance is one of the batch's contexts (a configured Simulation: mesh, source,
tally layout, run parameters) with its own optical properties, photon range and
tallies.  ``Batch.run()`` zeroes every instance's tallies and traces all instances in
one launch, replayed as a CUDA graph; the launch configuration (threads per block,
resident blocks per SM, BVH stack depth) is picked by the autotuner on the first run
unless fixed with ``set_config``.  Each instance's tallies equal those of
``Simulation.run`` on its context with its media and photon range, bit for bit.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import List, Sequence

import numpy as np

from . import _native as N
from .propagation import Simulation, gradient_dict, tallies_dict


@dataclass
class Instance:
    context: int                # index into the batch's simulations
    nmuasg: np.ndarray          # [R, 4] n, mua, mus, g (R <= 8)
    n_photons: int
    first: int = 0


def config_table() -> List[dict]:
    """The launch configurations the autotuner chooses from."""
    L = N.lib()
    out = []
    for k in range(L.lp_batch_config_count()):
        a, b, c = C.c_int32(), C.c_int32(), C.c_int32()
        N.check(L.lp_batch_config_info(k, C.byref(a), C.byref(b), C.byref(c)))
        out.append({"block": a.value, "min_blocks": b.value, "stack": c.value})
    return out


class Batch:
    def __init__(self, sims: Sequence[Simulation]):
        self._L = N.lib()
        self._sims = list(sims)          # keep the contexts alive as long as the batch
        arr = (C.c_void_p * len(sims))(*[s._h.value for s in sims])
        h = C.c_void_p()
        N.check(self._L.lp_batch_create(C.byref(h), len(sims), arr))
        self._h = h
        self._inst: List[Instance] = []
        self._geo = sims[0].geometry()

    def close(self):
        if getattr(self, "_h", None):
            self._L.lp_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _ck(self, rc):
        N.check_batch(rc, self._h)

    def set_instances(self, instances: Sequence[Instance]):
        arr = (N.Instance * max(len(instances), 1))()
        for i, x in enumerate(instances):
            nm = np.asarray(x.nmuasg, np.float32).reshape(-1, 4)
            arr[i].context = int(x.context)
            arr[i].n_media = nm.shape[0]
            for k, v in enumerate(nm.ravel()[: 4 * N.BATCH_MAX_MEDIA]):
                arr[i].nmuasg[k] = float(v)
            arr[i].first = int(x.first)
            arr[i].n_photons = int(x.n_photons)
        self._ck(self._L.lp_batch_set_instances(self._h, len(instances), arr))
        self._inst = list(instances)

    def set_gradient(self, enable: bool):
        self._ck(self._L.lp_batch_set_gradient(self._h, 1 if enable else 0))

    def set_plain_threshold(self, photons: int):
        """Instances of at least `photons` photons run as a transport launch of their own
        inside the batch's graph (<= 0: all share the batch launch; default 2^20)."""
        self._ck(self._L.lp_batch_set_plain_threshold(self._h, int(photons)))

    def plain_count(self) -> int:
        """Instances the current setting runs as launches of their own."""
        n = C.c_int32()
        self._ck(self._L.lp_batch_plain_count(self._h, C.byref(n)))
        return n.value

    def set_config(self, config: int):
        self._ck(self._L.lp_batch_set_config(self._h, int(config)))

    def autotune(self, photons: int = 4_000_000):
        """Time every eligible configuration; returns (best, ns per photon per config)."""
        k = self._L.lp_batch_config_count()
        ns = np.zeros(k, np.float64)
        best = C.c_int32()
        self._ck(self._L.lp_batch_autotune(self._h, int(photons), C.byref(best),
                                           ns.ctypes.data_as(C.POINTER(C.c_double))))
        return best.value, ns

    def run(self):
        self._ck(self._L.lp_batch_run(self._h))

    def last_ms(self) -> float:
        ms = C.c_float()
        self._ck(self._L.lp_batch_last_ms(self._h, C.byref(ms)))
        return float(ms.value)

    def ring_signals(self):
        """(S [n_inst, n_det], relative standard error [n_inst, n_det])."""
        d = max(1, self._sims[0].geometry_rings().shape[0])
        n = max(1, len(self._inst))
        s = np.zeros((n, d), np.float64)
        e = np.zeros((n, d), np.float64)
        dp = C.POINTER(C.c_double)
        self._ck(self._L.lp_batch_ring_signals(self._h, s.ctypes.data_as(dp), e.ctypes.data_as(dp)))
        nd = self._sims[0].geometry_rings().shape[0]
        return s[: len(self._inst), :nd], e[: len(self._inst), :nd]

    def tallies(self, i: int) -> dict:
        T = N.Tallies()
        self._ck(self._L.lp_batch_get_tallies(self._h, int(i), C.byref(T)))
        return tallies_dict(T, self._geo)

    def gradient(self, i: int) -> dict:
        g = N.Gradient()
        self._ck(self._L.lp_batch_get_gradient(self._h, int(i), C.byref(g)))
        return gradient_dict(g)
