"""Python interface to the B200 transport library.

Two layers:

``Simulation``
    A thin owner of one ``lp_ctx`` (one GPU, one CUDA stream) with numpy in/out.

``CalculatePropagation``
    The launcher interface of the reference, src/Simulation/CalculatePropagation.hpp:212-388,
    with the same method names, argument order and call sequence
    (setters -> Init() -> Propagation() -> Get*Image()).  VTK types become numpy
    arrays and ``ImageData`` (a minimal vtkImageData with VTK-style extents).
    Methods return the reference's status codes (0 == SUCCESS).
"""
from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

from . import _native as N

SUCCESS, FAILURE = 0, 1
# component ids of the SFT / RTd images (Rxy_Log_SURF / _FETAL / _TRANS in the reference)
RXY_LOG_SURF, RXY_LOG_FETAL, RXY_LOG_TRANS = 0, 1, 2


def _f32(a, n=None):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float32).ravel())
    if n is not None and a.size != n:
        raise ValueError(f"expected {n} floats, got {a.size}")
    return a


def _i32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32).ravel())


def tallies_dict(T: N.Tallies, g: N.Geometry) -> dict:
    """Copy an lp_tallies into numpy arrays shaped like the reference's images."""

    def arr(p, n, shape):
        if n == 0:
            return np.zeros(shape, np.uint64)
        return np.ctypeslib.as_array(p, shape=(n,)).copy().reshape(shape)

    return {
        "sft": arr(T.sft, g.sft_nx * g.sft_ny * 3, (g.sft_ny, g.sft_nx, 3)),
        "rtd": arr(T.rtd, g.dimR * g.dimAlpha * 3, (g.dimAlpha, g.dimR, 3)),
        "rz": arr(T.rz, g.rz_nr * g.rz_nz * 2, (g.rz_nz, g.rz_nr, 2)),
        "vox": arr(T.vox, T.n_vox, (T.n_vox,)),
        "rbins": arr(T.rbins, T.n_rbins * 2, (T.n_rbins, 2)),
        "region": arr(T.region, T.n_region, (T.n_region,)),
        "det": arr(T.det, T.n_det * 2, (T.n_det, 2)),
        "counters": {k: int(T.counters[i]) for i, k in enumerate(N.COUNTER_NAMES)},
    }


def gradient_dict(g: N.Gradient) -> dict:
    D, R = g.n_det, g.n_media

    def arr(p, shape):
        n = int(np.prod(shape))
        return np.ctypeslib.as_array(p, shape=(n,)).copy().reshape(shape) if n else np.zeros(shape)

    return {"n_photons": int(g.n_photons), "signal": arr(g.signal, (D,)), "signal_se": arr(g.signal_se, (D,)),
            "d_mua": arr(g.d_mua, (D, R)), "d_mus": arr(g.d_mus, (D, R)),
            "d_mua_se": arr(g.d_mua_se, (D, R)), "d_mus_se": arr(g.d_mus_se, (D, R))}


class Simulation:
    """One transport context on one GPU."""

    def __init__(self, device: int = 0):
        L = N.lib()
        h = C.c_void_p()
        N.check(L.lp_create(C.byref(h), device))
        self._h = h
        self._L = L
        self.device = device
        self._n_media = 0
        self._rings = np.zeros((0, 2), np.float32)

    # -- lifetime
    def close(self):
        if getattr(self, "_h", None):
            self._L.lp_destroy(self._h)
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
        N.check(rc, self._h)

    # -- inputs
    def set_mesh(self, tri, nrm, med):
        tri, nrm, med = _f32(tri), _f32(nrm), _i32(med)
        n = tri.size // 9
        if tri.size != 9 * n or nrm.size != 3 * n or med.size != 2 * n:
            raise ValueError("mesh arrays must be [T,9], [T,3], [T,2]")
        self._ck(self._L.lp_set_mesh(self._h, n, N.fptr(tri), N.fptr(nrm), N.iptr(med)))

    def set_media(self, nmuasg):
        a = _f32(nmuasg)
        self._ck(self._L.lp_set_media(self._h, a.size // 4, N.fptr(a)))
        self._n_media = a.size // 4

    def set_source(self, p_start, v_start, ep0xyz, v_occ=None):
        p, v, e = _f32(p_start, 3), _f32(v_start), _f32(ep0xyz, 12)
        occ = _i32(v_occ if v_occ is not None else [1] * (v.size // 3))
        self._ck(self._L.lp_set_source(self._h, N.fptr(p), N.fptr(v), N.iptr(occ), v.size // 3, N.fptr(e)))

    def set_fiber_source(self, radius: float, na: float):
        self._ck(self._L.lp_set_fiber_source(self._h, float(radius), float(na)))

    def set_tally_grid(self, dimensions, det_grid, fetal_id: int):
        d, g = _f32(dimensions, 3), _f32(det_grid, 6)
        self._ck(self._L.lp_set_tally_grid(self._h, N.fptr(d), N.fptr(g), int(fetal_id)))

    def set_params(self, chance, w_threshold, factor=1.0, seed=0x4C50, compat=N.COMPAT_ALL):
        self._ck(self._L.lp_set_params(self._h, chance, w_threshold, factor, seed, compat))

    def set_extra_tallies(self, vox_n=(0, 0, 0), vox_d=(1, 1, 1), n_rbins=0, rbin_dr=1.0, det_r=None):
        vn, vd = _i32(vox_n), _f32(vox_d, 3)
        dr = _f32(det_r if det_r is not None else np.zeros((0, 2)))
        self._ck(self._L.lp_set_extra_tallies(self._h, N.iptr(vn), N.fptr(vd), int(n_rbins), float(rbin_dr),
                                              dr.size // 2, N.fptr(dr)))
        self._rings = dr.reshape(-1, 2).copy()

    def set_arithmetic(self, exact: bool):
        """exact=True: the reference kernel's operation order; False (default): fast."""
        self._ck(self._L.lp_set_arithmetic(self._h, 1 if exact else 0))

    def set_safety_grid(self, max_cells: int):
        """Cells of the query-skipping safety grid (0 disables it; results are unchanged)."""
        self._ck(self._L.lp_set_safety_grid(self._h, int(max_cells)))

    # -- differentiation (lp_set_gradient / lp_forward / lp_backward)
    def set_gradient(self, enable: bool):
        """Accumulate d(ring signal)/d(mua, mus) sums in the following runs."""
        self._ck(self._L.lp_set_gradient(self._h, 1 if enable else 0))

    def gradient(self) -> dict:
        """Ring signals S_d and dS_d/dmua_r, dS_d/dmus_r with standard errors."""
        g = N.Gradient()
        self._ck(self._L.lp_get_gradient(self._h, C.byref(g)))
        return gradient_dict(g)

    def forward(self, n: int, first: int = 0) -> np.ndarray:
        """Zero the tallies, trace photons [first, first + n) with differentiation on and
        return the ring signals."""
        d = max(1, len(self.geometry_rings()))
        out = np.zeros(d, np.float64)
        self._ck(self._L.lp_forward(self._h, int(first), int(n), out.ctypes.data_as(C.POINTER(C.c_double))))
        return out[:len(self.geometry_rings())]

    def backward(self, grad_signal):
        """Vector-Jacobian product of the last forward: (grad_mua, grad_mus) per region."""
        g = np.ascontiguousarray(grad_signal, np.float64)
        r = self._n_media
        gm, gs = np.zeros(r, np.float64), np.zeros(r, np.float64)
        dp = C.POINTER(C.c_double)
        self._ck(self._L.lp_backward(self._h, g.ctypes.data_as(dp), gm.ctypes.data_as(dp), gs.ctypes.data_as(dp)))
        return gm, gs

    def geometry_rings(self) -> np.ndarray:
        return self._rings

    def set_cell_lists(self, enable: bool):
        """Cells touched by triangles list them for short-step queries (default on;
        results are unchanged either way)."""
        self._ck(self._L.lp_set_cell_lists(self._h, 1 if enable else 0))

    def set_cell_margin(self, cells: float):
        """Margin of the cell lists in cells (default 0.5): each list holds the triangles
        touching its cell widened by this much (results are unchanged)."""
        self._ck(self._L.lp_set_cell_margin(self._h, float(cells)))

    def set_tally_aggregation(self, enable: bool):
        """Sum same-cell absorption deposits across the warp before the atomic adds
        (tallies are identical either way)."""
        self._ck(self._L.lp_set_tally_aggregation(self._h, 1 if enable else 0))

    def set_smem_budget(self, nbytes: int):
        """Shared memory per block for staged BVH nodes and triangles (the rest is L1)."""
        self._ck(self._L.lp_set_smem_budget(self._h, int(nbytes)))

    def set_max_steps(self, n: int):
        self._ck(self._L.lp_set_max_steps(self._h, int(n)))

    def set_exit_records(self, capacity: int):
        self._ck(self._L.lp_set_exit_records(self._h, int(capacity)))

    # -- run
    def run(self, n: int, first: int = 0):
        self._ck(self._L.lp_run(self._h, int(first), int(n)))

    def run_async(self, n: int, first: int = 0):
        self._ck(self._L.lp_run_async(self._h, int(first), int(n)))

    def sync(self):
        self._ck(self._L.lp_sync(self._h))

    def zero(self):
        self._ck(self._L.lp_zero_tallies(self._h))

    def kernel_ms(self) -> float:
        ms = C.c_float()
        self._ck(self._L.lp_last_kernel_ms(self._h, C.byref(ms)))
        return float(ms.value)

    # -- outputs
    def geometry(self) -> N.Geometry:
        g = N.Geometry()
        self._ck(self._L.lp_get_geometry(self._h, C.byref(g)))
        return g

    def tallies(self) -> dict:
        """Fixed-point (2^32 per unit weight) uint64 tallies, copied out."""
        g = self.geometry()
        T = N.Tallies()
        self._ck(self._L.lp_get_tallies(self._h, C.byref(T)))
        return tallies_dict(T, g)

    # -- checkpoint / resume (lp_set_tallies, lp_get/set_gradient_sums)
    def checkpoint(self) -> dict:
        """The integer tallies, the counters and the differentiation sums.  With the seed
        and the id of the next photon that is all a resumed run needs: photon streams
        depend on the seed and the photon id alone."""
        g = self.geometry()
        T = N.Tallies()
        self._ck(self._L.lp_get_tallies(self._h, C.byref(T)))
        t = tallies_dict(T, g)
        ck = {k: t[k].copy() for k in ("sft", "rtd", "rz", "vox", "rbins", "region", "det")}
        ck["counters"] = np.array([T.counters[i] for i in range(N.NCOUNTERS)], np.uint64)
        n = int(t["det"].shape[0]) * self._n_media * 5
        ck["grad"] = np.zeros(n, np.float64)
        if n:
            self._ck(self._L.lp_get_gradient_sums(self._h, ck["grad"].ctypes.data_as(C.POINTER(C.c_double)), n))
        return ck

    def restore(self, ck: dict):
        """Replace this context's tallies, counters and differentiation sums by a checkpoint
        taken with the same tally layout."""
        arrs = {k: np.ascontiguousarray(ck[k], np.uint64) for k in ("sft", "rtd", "rz", "vox", "rbins", "region",
                                                                    "det")}
        T = N.Tallies()
        for k, a in arrs.items():
            setattr(T, k, a.ctypes.data_as(C.POINTER(C.c_uint64)))
        for i in range(N.NCOUNTERS):
            T.counters[i] = int(ck["counters"][i])
        T.n_vox, T.n_rbins = arrs["vox"].size, arrs["rbins"].shape[0]
        T.n_region, T.n_det = arrs["region"].size, arrs["det"].shape[0]
        self._ck(self._L.lp_set_tallies(self._h, C.byref(T)))
        g = np.ascontiguousarray(ck.get("grad", np.zeros(0)), np.float64)
        if g.size:
            self._ck(self._L.lp_set_gradient_sums(self._h, g.ctypes.data_as(C.POINTER(C.c_double)), g.size))

    def stats(self) -> dict:
        st = N.Stats()
        self._ck(self._L.lp_get_stats(self._h, C.byref(st)))
        return {k: getattr(st, k) for k, _ in N.Stats._fields_}

    def device_tallies(self) -> N.DeviceTallies:
        d = N.DeviceTallies()
        self._ck(self._L.lp_get_device_tallies(self._h, C.byref(d)))
        return d

    def exit_records(self, n: int) -> np.ndarray:
        out = np.zeros((n, 8), np.float32)
        self._ck(self._L.lp_get_exit_records(self._h, N.fptr(out), int(n)))
        return out

    def query(self, orig, dirs, ref=None, t_max=None):
        o, d = _f32(orig), _f32(dirs)
        n = o.size // 3
        r = _i32(ref if ref is not None else np.full(n, -1))
        tm = _f32(t_max if t_max is not None else np.full(n, 10000.0))
        ids = np.zeros(n, np.int32)
        ts = np.zeros(n, np.float32)
        self._ck(self._L.lp_query_triangles(self._h, n, N.fptr(o), N.fptr(d), N.iptr(r), N.fptr(tm),
                                            N.iptr(ids), N.fptr(ts)))
        return ids, ts


def fp32_peak_tflops(device: int = 0) -> float:
    """Measured FP32 FMA throughput of the device (TFLOP/s)."""
    t = C.c_double()
    N.check(N.lib().lp_fp32_peak(device, C.byref(t)))
    return float(t.value)


def l2_atomic_peak(device: int = 0) -> float:
    """Measured throughput of 64-bit atomic adds to an L2-resident buffer (atomics/s)."""
    t = C.c_double()
    N.check(N.lib().lp_l2_atomic_peak(device, C.byref(t)))
    return float(t.value)


def philox_blocks(ctr, key, n, device=0) -> np.ndarray:
    """n Philox4x32-10 blocks computed on the GPU, counter word 2 incremented per block."""
    c = np.ascontiguousarray(ctr, np.uint32)
    k = np.ascontiguousarray(key, np.uint32)
    out = np.zeros((n, 4), np.uint32)
    N.check(N.lib().lp_philox_blocks(device, N.u32ptr(c), N.u32ptr(k), n, N.u32ptr(out)))
    return out


@dataclass
class ImageData:
    """Minimal stand-in for vtkImageData: a 2-D extent with float components."""
    extent: tuple
    data: np.ndarray   # [ny, nx, ncomp], indexed [j - extent[2], i - extent[0], c]

    def GetExtent(self):
        return tuple(self.extent)

    def GetDimensions(self):
        return (self.data.shape[1], self.data.shape[0], 1)

    def GetNumberOfScalarComponents(self):
        return self.data.shape[2]

    def GetScalarComponentAsFloat(self, i, j, k, c):
        return float(self.data[j - self.extent[2], i - self.extent[0], c])

    def SetScalarComponentFromFloat(self, i, j, k, c, v):
        self.data[j - self.extent[2], i - self.extent[0], c] = v

    def component(self, c) -> "ImageData":
        return ImageData(self.extent, self.data[:, :, c:c + 1].copy())


class CalculatePropagation:
    """Launcher with the reference's interface (CalculatePropagation.hpp:212-388)."""

    def __init__(self, device: int = 0):
        self._device = device
        self.verbose = False
        self.showPercent = False
        self.numberPhotons = 1
        self.numPhotonInteractions = 100
        self.chance = 0.5                  # constructor defaults, CalculatePropagation.cpp:27-79
        self.w_threshold = 0.001
        self.pixelPerUnitFactor = 100.0
        self.fetalTissueID = 1
        self.DetGridDims = [1.0] * 6
        self.eP0XYZ = [0.0] * 12
        self.eP0XYZ[3], self.eP0XYZ[7], self.eP0XYZ[11] = 1.0, 1.0, 1.0
        self.dimensions = None
        self.nmuasG = None
        self.triangles = None
        self.normals = None
        self.triN = None
        self.vStart, self.vStartOcc, self.pStart = None, None, None
        self.seed = 0x4C50
        self.exact = False                 # reference-order arithmetic (lp_set_arithmetic)
        self.compat = N.COMPAT_ALL
        self.extra = None
        self._sim: Optional[Simulation] = None
        self._images = None
        self.neededTime_ms = 0.0

    # -- setters (CalculatePropagation.cpp:249-777)
    def SetVerbosity(self, verb): self.verbose = bool(verb)
    def SetShowPercentDone(self, s): self.showPercent = bool(s)
    def SetDeviceType(self, device: int):
        if device == 0:
            raise ValueError("SetDeviceType(0): this build runs on the GPU only")
    def SetNumberOfPhotonInteractions(self, n): self.numPhotonInteractions = int(n)
    def SetNumberOfPhotons(self, n): self.numberPhotons = int(n)
    def SetChanceForRoulette(self, c): self.chance = float(c)
    def SetWeightThreshold(self, w): self.w_threshold = float(w)
    def SetPixelPerUnitFactor(self, f): self.pixelPerUnitFactor = float(f)
    def SetFetalTissueID(self, i): self.fetalTissueID = int(i)
    def SetDimensions(self, dims): self.dimensions = [float(x) for x in dims]
    def SetSeed(self, seed): self.seed = int(seed)
    def SetArithmetic(self, exact): self.exact = bool(exact)
    def SetCompat(self, compat): self.compat = int(compat)

    def SetDetectionGridDimensions(self, *grid):
        g = grid[0] if len(grid) == 1 else grid
        self.DetGridDims = [float(x) for x in g]

    def SetTissueProperties(self, refractionInd, absorbtionCoeffs, anisotropies, scatterCoeffs):
        # packs n, mua, mus, g per region (CalculatePropagation.cpp:427-451)
        n = len(refractionInd)
        a = np.zeros((n, 4), np.float32)
        a[:, 0], a[:, 1], a[:, 2], a[:, 3] = refractionInd, absorbtionCoeffs, scatterCoeffs, anisotropies
        self.nmuasG = a

    def SetTriangles(self, tri): self.triangles = np.asarray(tri, np.float32).reshape(-1, 9)
    def SetNormals(self, nrm): self.normals = np.asarray(nrm, np.float32).reshape(-1, 3)
    def SetInnerAndOuterTissueIndices(self, med): self.triN = np.asarray(med, np.int32).reshape(-1, 2)

    def SetStartTrajectories(self, trajectories, trajOcc):
        self.vStart = np.asarray(trajectories, np.float32).ravel()
        self.vStartOcc = np.asarray(trajOcc, np.int32).ravel()

    def SetStartTrajectory(self, *v):
        self.vStart = np.asarray(v[0] if len(v) == 1 else v, np.float32).ravel()

    def SetStartPoint(self, *p):
        self.pStart = np.asarray(p[0] if len(p) == 1 else p, np.float32).ravel()

    def SetPOI(self, *p):
        p = p[0] if len(p) == 1 else p
        self.eP0XYZ[0:3] = [float(x) for x in p]

    def SetExVector(self, x, y, z): self.eP0XYZ[3:6] = [x, y, z]
    def SetEyVector(self, x, y, z): self.eP0XYZ[6:9] = [x, y, z]
    def SetEzVector(self, x, y, z): self.eP0XYZ[9:12] = [x, y, z]

    def SetBasisVectors(self, veX, veY, veZ):
        self.SetExVector(*veX)
        self.SetEyVector(*veY)
        self.SetEzVector(*veZ)

    def SetExtraTallies(self, vox_n=(0, 0, 0), vox_d=(1, 1, 1), n_rbins=0, rbin_dr=1.0, det_r=None):
        self.extra = dict(vox_n=vox_n, vox_d=vox_d, n_rbins=n_rbins, rbin_dr=rbin_dr, det_r=det_r)

    # -- getters
    def GetNumberOfPhotons(self): return self.numberPhotons
    def GetChanceForRoulette(self): return self.chance
    def GetWeightThreshold(self): return self.w_threshold
    def GetStartPoint(self): return None if self.pStart is None else self.pStart.tolist()
    def GetStartTrajectory(self): return None if self.vStart is None else self.vStart.tolist()

    # -- Init / Propagation (CalculatePropagation.cpp:2003-2025)
    def Init(self) -> int:
        if self._sim is None:
            self._sim = Simulation(self._device)
        s = self._sim
        s.set_mesh(self.triangles, self.normals, self.triN)
        s.set_media(self.nmuasG)
        s.set_source(self.pStart, self.vStart, self.eP0XYZ, self.vStartOcc)
        s.set_tally_grid(self.dimensions, self.DetGridDims, self.fetalTissueID)
        s.set_params(self.chance, self.w_threshold, self.pixelPerUnitFactor, self.seed, self.compat)
        s.set_arithmetic(self.exact)
        if self.extra:
            s.set_extra_tallies(**self.extra)
        s.zero()
        return SUCCESS

    def Propagation(self) -> int:
        if self._sim is None:
            return FAILURE
        t0 = time.perf_counter()
        self._sim.run(self.numberPhotons)
        self.neededTime_ms = self._sim.kernel_ms()
        self._tallies = self._sim.tallies()
        self._host_ms = (time.perf_counter() - t0) * 1e3
        self._build_images()
        return SUCCESS

    def _build_images(self):
        g = self._sim.geometry()
        t = self._tallies
        sc = 1.0 / N.FIX_ONE
        hx, hy = g.dimx // 2, g.dimy // 2
        self._sft = ImageData((-hx, hx, -hy, hy, 0, 0), (t["sft"] * sc).astype(np.float32))
        rtd = np.transpose(t["rtd"], (0, 1, 2))   # [alpha][r][c] -> image [j=alpha][i=r][c]
        self._rtd = ImageData((0, g.dimR - 1, 0, g.dimAlpha - 1, 0, 0), (rtd * sc).astype(np.float32))
        # r-z image extent [-dimR, dimR] x [-dimz, 0]; row z (depth cz) sits at j = -cz
        rz = (t["rz"] * sc).astype(np.float32)[::-1]
        self._arz = ImageData((-g.dimR, g.dimR, -g.dimz, 0, 0, 0), rz)

    def GetSFTImage(self, component: Optional[int] = None) -> ImageData:
        return self._sft if component is None else self._sft.component(component)

    def GetRTdImage(self, component: Optional[int] = None) -> ImageData:
        return self._rtd if component is None else self._rtd.component(component)

    def GetArzImage(self) -> ImageData:
        return self._arz.component(0)

    def GetPhirzImage(self) -> ImageData:
        return self._arz.component(1)

    def GetTallies(self) -> dict:
        return self._tallies

    def PrintTimeSpent(self):
        print("############# Calculation Time #############")
        print(f"Time in ms: {self.neededTime_ms} \t| Time in s: {self.neededTime_ms / 1e3}")

    def PrintSimulationParams(self):
        print("########### Simulation Parameter ###########")
        print("Device Name: CUDA device", self._device)
        print("Number of Photons:", self.numberPhotons)
