"""ctypes wrapper around the CPU oracle (oracle/_build/liblporacle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by the smoke check and by the CPU
baseline leg of bench.py, never by the lightpropagation_b200 package.

Also wraps oracle/_ref/libclref.so, the reference kernel compiled for the CPU by
oracle/build_ref.py, when that library has been built.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liblporacle.so")
REF_PATH = os.path.join(HERE, "_ref", "libclref.so")

RNG_RAN3_SHARED, RNG_RAN3_PHOTON, RNG_PHILOX = 0, 1, 2
COMPAT_EXIT_RSP, COMPAT_AXIS_NORMAL, COMPAT_SIGNED_FRESNEL = 1, 2, 4
COMPAT_ALL = 7
NCOUNTERS = 16
COUNTER_NAMES = ["scatter", "boundary", "query", "roulette", "miss", "capped",
                 "rz_drop", "vox_drop", "photons", "draws", "region_mismatch"]
FIX_SCALE = float(2 ** 32)

_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int32)
_up = C.POINTER(C.c_uint64)


class Problem(C.Structure):
    _fields_ = [
        ("n_tri", C.c_int32), ("tri", _fp), ("nrm", _fp), ("med", _ip),
        ("n_media", C.c_int32), ("nmuasg", _fp),
        ("p_start", C.c_float * 3), ("v_start", C.c_float * 3), ("ep0xyz", C.c_float * 12),
        ("dimensions", C.c_float * 3), ("det_grid", C.c_float * 6),
        ("fetal_id", C.c_int32), ("chance", C.c_float), ("w_threshold", C.c_float),
        ("factor", C.c_float),
        ("compat", C.c_uint32), ("rng_mode", C.c_int32), ("seed", C.c_uint64),
        ("stream", C.c_uint32), ("max_steps", C.c_int64),
        ("vox_n", C.c_int32 * 3), ("vox_d", C.c_float * 3),
        ("n_rbins", C.c_int32), ("rbin_dr", C.c_float),
        ("n_det", C.c_int32), ("det_r", _fp),
        ("src_type", C.c_int32), ("src_radius", C.c_float), ("src_cos_max", C.c_float),
    ]


class Geometry(C.Structure):
    _fields_ = [(n, C.c_int32) for n in
                ("dimx", "dimy", "dimz", "dimR", "dimAlpha", "sft_nx", "sft_ny",
                 "rz_nr", "rz_nz", "kernel_dimR")]


class Tallies(C.Structure):
    _fields_ = [
        ("sft", _up), ("rtd", _up), ("rz", _up), ("vox", _up), ("rbins", _up),
        ("region", _up), ("det", _up), ("counters", C.c_uint64 * NCOUNTERS),
        ("exit_rec", _fp), ("rz_ref", _fp), ("rz_ref_cells", C.c_int64),
        ("rz_ref_offset", C.c_int64), ("grad", C.POINTER(C.c_double)),
    ]


_lib = None
_ref = None


def build() -> None:
    subprocess.check_call(["make", "-s", "-C", HERE])


def lib():
    global _lib
    if _lib is None:
        if not os.path.isfile(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        L.lpo_run.argtypes = [C.POINTER(Problem), C.c_int64, C.c_int64, C.c_int,
                              _fp, _ip, C.POINTER(Tallies)]
        L.lpo_run.restype = C.c_int
        L.lpo_philox4x32_10.argtypes = [C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                        C.POINTER(C.c_uint32)]
        L.lpo_ran3_init.argtypes = [C.c_int32, _fp, _ip]
        L.lpo_ran3_draw.argtypes = [_fp, _ip]
        L.lpo_ran3_draw.restype = C.c_float
        L.lpo_geometry_of.argtypes = [_fp, _fp, C.POINTER(Geometry)]
        L.lpo_rspecular.argtypes = [_fp]
        L.lpo_rspecular.restype = C.c_float
        L.lpo_fresnel.argtypes = [C.c_float, C.c_float, C.c_float]
        L.lpo_fresnel.restype = C.c_float
        L.lpo_hg_cos_theta.argtypes = [C.c_float, C.c_float]
        L.lpo_hg_cos_theta.restype = C.c_float
        L.lpo_find_triangle.argtypes = [_fp, C.c_int32, C.c_int32, _fp, _fp, _fp]
        L.lpo_find_triangle.restype = C.c_int32
        L.lpo_fix.argtypes = [C.c_float]
        L.lpo_fix.restype = C.c_uint64
        _dp = C.POINTER(C.c_double)
        L.lpo64_mesh_build.argtypes = [_fp, C.c_int32]
        L.lpo64_mesh_build.restype = C.c_void_p
        L.lpo64_mesh_free.argtypes = [C.c_void_p]
        L.lpo64_mesh_query.argtypes = [C.c_void_p, C.c_int32, _dp, _dp, C.c_double, _dp]
        L.lpo64_mesh_query.restype = C.c_int32
        L.lpo64_find_triangle.argtypes = [_fp, C.c_int32, C.c_int32, _dp, _dp, C.c_double, _dp]
        L.lpo64_find_triangle.restype = C.c_int32
        L.lpo64_fresnel.argtypes = [C.c_double, C.c_double, C.c_double]
        L.lpo64_fresnel.restype = C.c_double
        L.lpo64_run.argtypes = [C.POINTER(Problem), C.c_void_p, C.c_int64, C.c_int64, C.c_int,
                                C.POINTER(Tallies)]
        L.lpo64_run.restype = C.c_int
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.isfile(REF_PATH)


def ref():
    global _ref
    if _ref is None:
        R = C.CDLL(REF_PATH)
        R.clref_psnr_state.argtypes = [C.c_int, _fp, _ip]
        R.clref_run.argtypes = [C.c_int, C.c_float, _fp, _ip, _fp, C.c_float, C.c_float,
                                C.c_int, _fp, _fp, _fp, _fp, _fp, _fp, _fp, _ip, _fp, _fp,
                                _ip, C.c_long]
        R.clref_run.restype = C.c_int
        R.clref_find_triangle.argtypes = [C.c_int, _fp, C.c_int, _fp, _fp, _fp]
        R.clref_find_triangle.restype = C.c_int
        R.clref_fresnel.argtypes = [C.c_float, C.c_float, C.c_float]
        R.clref_fresnel.restype = C.c_float
        _ref = R
    return _ref


def fptr(a: np.ndarray):
    return a.ctypes.data_as(_fp)


def iptr(a: np.ndarray):
    return a.ctypes.data_as(_ip)


def uptr(a: np.ndarray):
    return a.ctypes.data_as(_up)


@dataclass
class Case:
    """One transport problem in the reference's layouts (see lp_oracle.h)."""
    tri: np.ndarray            # float32 [T, 9]
    nrm: np.ndarray            # float32 [T, 3]
    med: np.ndarray            # int32   [T, 2]
    nmuasg: np.ndarray         # float32 [R, 4]
    p_start: np.ndarray        # float32 [3]
    v_start: np.ndarray        # float32 [3]
    ep0xyz: np.ndarray         # float32 [12]
    dimensions: np.ndarray     # float32 [3]
    det_grid: np.ndarray       # float32 [6]
    fetal_id: int = 1
    chance: float = 0.1
    w_threshold: float = 1e-4
    factor: float = 1.0
    vox_n: tuple = (0, 0, 0)
    vox_d: tuple = (1.0, 1.0, 1.0)
    n_rbins: int = 0
    rbin_dr: float = 1.0
    det_r: Optional[np.ndarray] = None   # float32 [D, 2]
    src_type: int = 0
    src_radius: float = 0.0
    src_cos_max: float = 1.0
    keep: list = field(default_factory=list, repr=False)

    def problem(self, rng_mode=RNG_PHILOX, seed=0x4C50, compat=COMPAT_ALL, stream=0,
                max_steps=0) -> Problem:
        P = Problem()
        arrs = [np.ascontiguousarray(self.tri, np.float32), np.ascontiguousarray(self.nrm, np.float32),
                np.ascontiguousarray(self.med, np.int32), np.ascontiguousarray(self.nmuasg, np.float32)]
        det_r = np.ascontiguousarray(self.det_r if self.det_r is not None else np.zeros((0, 2)), np.float32)
        self.keep = arrs + [det_r]
        P.n_tri = arrs[0].shape[0]
        P.tri, P.nrm, P.med = fptr(arrs[0]), fptr(arrs[1]), iptr(arrs[2])
        P.n_media = arrs[3].shape[0]
        P.nmuasg = fptr(arrs[3])
        P.p_start[:] = [float(x) for x in self.p_start]
        P.v_start[:] = [float(x) for x in self.v_start]
        P.ep0xyz[:] = [float(x) for x in self.ep0xyz]
        P.dimensions[:] = [float(x) for x in self.dimensions]
        P.det_grid[:] = [float(x) for x in self.det_grid]
        P.fetal_id = int(self.fetal_id)
        P.chance, P.w_threshold, P.factor = self.chance, self.w_threshold, self.factor
        P.compat, P.rng_mode, P.seed, P.stream, P.max_steps = compat, rng_mode, seed, stream, max_steps
        P.vox_n[:] = list(self.vox_n)
        P.vox_d[:] = list(self.vox_d)
        P.n_rbins, P.rbin_dr = self.n_rbins, self.rbin_dr
        P.n_det = det_r.shape[0]
        P.det_r = fptr(det_r)
        P.src_type, P.src_radius, P.src_cos_max = self.src_type, self.src_radius, self.src_cos_max
        return P


def geometry(case: Case) -> Geometry:
    g = Geometry()
    d = np.asarray(case.dimensions, np.float32)
    dg = np.asarray(case.det_grid, np.float32)
    lib().lpo_geometry_of(fptr(d), fptr(dg), C.byref(g))
    return g


@dataclass
class Result:
    sft: np.ndarray
    rtd: np.ndarray
    rz: np.ndarray
    vox: np.ndarray
    rbins: np.ndarray
    region: np.ndarray
    det: np.ndarray
    counters: dict
    exit_rec: Optional[np.ndarray] = None
    rz_ref: Optional[np.ndarray] = None
    ran3_state: Optional[np.ndarray] = None
    ran3_inext: Optional[np.ndarray] = None
    grad: Optional[np.ndarray] = None       # [n_det, n_media, 5] perturbation-MC sums


def gradient(res: Result, case: "Case", n: int):
    """Ring signals and their derivatives from the perturbation-MC sums of a run of n
    photons (see lpo_tallies.grad): (S [D], dS/dmua [D, R], dS/dmus [D, R])."""
    s = res.det[:, 0].astype(np.float64) / 2.0 ** 32 / n
    g = res.grad
    f = float(case.factor)
    mus = np.asarray(case.nmuasg, np.float64)[:, 2]
    d_mua = -g[:, :, 0] / f / n
    with np.errstate(divide="ignore", invalid="ignore"):
        d_mus = np.where(mus > 0, (g[:, :, 1] / mus - g[:, :, 0] / f) / n, 0.0)
    return s, d_mua, d_mus


def run(case: Case, n: int, first: int = 0, rng_mode=RNG_PHILOX, seed=0x4C50,
        compat=COMPAT_ALL, nthreads=0, stream=0, exit_records=False, ran3_seed=None,
        ran3_state=None, rz_ref_pad=0, max_steps=0) -> Result:
    """Trace photons [first, first+n) on the CPU and return integer tallies."""
    g = geometry(case)
    P = case.problem(rng_mode, seed, compat, stream, max_steps)
    sft = np.zeros((g.sft_ny, g.sft_nx, 3), np.uint64)
    rtd = np.zeros((g.dimAlpha, g.dimR, 3), np.uint64)
    rz = np.zeros((g.rz_nz, g.rz_nr, 2), np.uint64)
    nv = int(np.prod(case.vox_n)) if case.vox_n[0] > 0 else 0
    vox = np.zeros((max(nv, 1),), np.uint64)
    rbins = np.zeros((max(case.n_rbins, 1), 2), np.uint64)
    region = np.zeros((case.nmuasg.shape[0],), np.uint64)
    ndet = 0 if case.det_r is None else case.det_r.shape[0]
    det = np.zeros((max(ndet, 1), 2), np.uint64)
    T = Tallies()
    T.sft, T.rtd, T.rz, T.vox = uptr(sft), uptr(rtd), uptr(rz), uptr(vox)
    T.rbins, T.region, T.det = uptr(rbins), uptr(region), uptr(det)
    grad = np.zeros((max(ndet, 1), case.nmuasg.shape[0], 5), np.float64)
    if ndet:
        T.grad = grad.ctypes.data_as(C.POINTER(C.c_double))
    rec = None
    if exit_records:
        rec = np.zeros((n, 8), np.float32)
        T.exit_rec = fptr(rec)
    rzref = None
    if rz_ref_pad > 0:
        cells = g.rz_nr * g.rz_nz
        rzref = np.zeros((cells + 2 * rz_ref_pad, 3), np.float32)
        T.rz_ref = fptr(rzref)
        T.rz_ref_cells = rzref.shape[0]
        T.rz_ref_offset = rz_ref_pad
    st = ix = None
    if rng_mode == RNG_RAN3_SHARED:
        if ran3_state is not None:
            st = np.array(ran3_state[0], np.float32).copy()
            ix = np.array(ran3_state[1], np.int32).copy()
        else:
            st, ix = ran3_init(1 if ran3_seed is None else ran3_seed)
    lib().lpo_run(C.byref(P), first, n, nthreads,
                  fptr(st) if st is not None else None, iptr(ix) if ix is not None else None,
                  C.byref(T))
    counters = {k: int(T.counters[i]) for i, k in enumerate(COUNTER_NAMES)}
    return Result(sft, rtd, rz, vox[:nv] if nv else vox[:0], rbins[:case.n_rbins], region,
                  det[:ndet], counters, rec, rzref, st, ix, grad[:ndet])


class Mesh64:
    """The FP64 oracle's bounding-volume tree over a mesh (float32 [T, 9] triangles)."""

    def __init__(self, tri):
        self.tri = np.ascontiguousarray(tri, np.float32).reshape(-1, 9)
        self.handle = lib().lpo64_mesh_build(fptr(self.tri), self.tri.shape[0])

    def query(self, p, v, ref_tri=-1, bound=10000.0):
        """(index or -1, distance) of the nearest triangle with 0 < t <= bound."""
        dp = C.POINTER(C.c_double)
        pp = np.ascontiguousarray(p, np.float64)
        vv = np.ascontiguousarray(v, np.float64)
        t = np.zeros(1, np.float64)
        j = lib().lpo64_mesh_query(self.handle, int(ref_tri), pp.ctypes.data_as(dp), vv.ctypes.data_as(dp),
                                   float(bound), t.ctypes.data_as(dp))
        return int(j), float(t[0])

    def brute(self, p, v, ref_tri=-1, bound=10000.0):
        """The same query by the brute-force scan."""
        dp = C.POINTER(C.c_double)
        pp = np.ascontiguousarray(p, np.float64)
        vv = np.ascontiguousarray(v, np.float64)
        t = np.zeros(1, np.float64)
        j = lib().lpo64_find_triangle(fptr(self.tri), self.tri.shape[0], int(ref_tri), pp.ctypes.data_as(dp),
                                      vv.ctypes.data_as(dp), float(bound), t.ctypes.data_as(dp))
        return int(j), float(t[0])

    def close(self):
        if self.handle:
            lib().lpo64_mesh_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass


def run64(case: Case, n: int, first: int = 0, seed=0x4C50, compat=COMPAT_ALL, nthreads=0, stream=0,
          exit_records=False, max_steps=0, mesh: Optional[Mesh64] = None) -> Result:
    """Trace photons [first, first+n) with the FP64 oracle (Philox draws, same tallies)."""
    g = geometry(case)
    P = case.problem(RNG_PHILOX, seed, compat, stream, max_steps)
    sft = np.zeros((g.sft_ny, g.sft_nx, 3), np.uint64)
    rtd = np.zeros((g.dimAlpha, g.dimR, 3), np.uint64)
    rz = np.zeros((g.rz_nz, g.rz_nr, 2), np.uint64)
    nv = int(np.prod(case.vox_n)) if case.vox_n[0] > 0 else 0
    vox = np.zeros((max(nv, 1),), np.uint64)
    rbins = np.zeros((max(case.n_rbins, 1), 2), np.uint64)
    region = np.zeros((case.nmuasg.shape[0],), np.uint64)
    ndet = 0 if case.det_r is None else case.det_r.shape[0]
    det = np.zeros((max(ndet, 1), 2), np.uint64)
    T = Tallies()
    T.sft, T.rtd, T.rz, T.vox = uptr(sft), uptr(rtd), uptr(rz), uptr(vox)
    T.rbins, T.region, T.det = uptr(rbins), uptr(region), uptr(det)
    grad = np.zeros((max(ndet, 1), case.nmuasg.shape[0], 5), np.float64)
    if ndet:
        T.grad = grad.ctypes.data_as(C.POINTER(C.c_double))
    rec = None
    if exit_records:
        rec = np.zeros((n, 8), np.float32)
        T.exit_rec = fptr(rec)
    rc = lib().lpo64_run(C.byref(P), mesh.handle if mesh is not None else None, first, n, nthreads, C.byref(T))
    if rc != 0:
        raise ValueError("lpo64_run: the FP64 oracle needs the Philox mode and at most 64 regions")
    counters = {k: int(T.counters[i]) for i, k in enumerate(COUNTER_NAMES)}
    return Result(sft, rtd, rz, vox[:nv] if nv else vox[:0], rbins[:case.n_rbins], region,
                  det[:ndet], counters, rec, None, None, None, grad[:ndet])


def ran3_init(seed: int):
    st = np.zeros(56, np.float32)
    ix = np.zeros(3, np.int32)
    lib().lpo_ran3_init(seed, fptr(st), iptr(ix))
    return st, ix


def philox(ctr, key):
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    lib().lpo_philox4x32_10(c, k, o)
    return list(o)


def ref_run(case: Case, n: int, ran3_seed: int, rz_pad: int):
    """Run the reference kernel (compiled for the CPU) on work-items 0..n-1."""
    R = ref()
    g = geometry(case)
    st = np.zeros(56, np.float32)
    ix = np.zeros(3, np.int32)
    R.clref_psnr_state(ran3_seed, fptr(st), iptr(ix))
    T = case.tri.shape[0]
    # one padding record in front of each mesh array so index -1 stays in bounds
    tri = np.zeros((T + 1) * 9, np.float32); tri[9:] = np.asarray(case.tri, np.float32).ravel()
    nrm = np.zeros((T + 1) * 3, np.float32); nrm[3:] = np.asarray(case.nrm, np.float32).ravel()
    med = np.zeros((T + 1) * 2, np.int32); med[2:] = np.asarray(case.med, np.int32).ravel()
    nm = np.ascontiguousarray(case.nmuasg, np.float32).ravel()
    vs = np.ascontiguousarray(case.v_start, np.float32)
    occ = np.array([n], np.int32)
    ps = np.ascontiguousarray(case.p_start, np.float32)
    sft = np.zeros((n, 8), np.float32)
    cells = g.rz_nr * g.rz_nz
    rz = np.zeros((cells + 2 * rz_pad, 3), np.float32)
    dims = np.array([g.dimx, g.dimy, g.dimz], np.float32)
    ep = np.ascontiguousarray(case.ep0xyz, np.float32)
    dg = np.ascontiguousarray(case.det_grid, np.float32)
    off = lambda a, k: C.cast(C.c_void_p(a.ctypes.data + k), _fp)
    R.clref_run(T, case.factor, fptr(vs), iptr(occ), fptr(ps), case.chance, case.w_threshold,
                case.fetal_id, fptr(sft), off(rz, rz_pad * 12), fptr(dims), fptr(ep), fptr(dg),
                off(tri, 36), off(nrm, 12), C.cast(C.c_void_p(med.ctypes.data + 8), _ip),
                fptr(nm), fptr(st), iptr(ix), n)
    return sft, rz, st, ix


def ref_ran3_state(seed: int):
    st = np.zeros(56, np.float32)
    ix = np.zeros(3, np.int32)
    ref().clref_psnr_state(seed, fptr(st), iptr(ix))
    return st, ix
