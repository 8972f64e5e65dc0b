"""ctypes bindings of liblpcuda.so (the C ABI declared in include/lpcuda.h).

The library is built in-tree by ``lightpropagation_b200.build.build()``.  There is
no fallback: if the shared library is missing or no GPU is present, calls raise.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblpcuda.so")

LP_OK = 0
ERRORS = {1: "invalid argument", 2: "CUDA error", 3: "call out of order", 4: "out of memory",
          5: "size out of range", 6: "device wait timed out"}
COMPAT_EXIT_RSP, COMPAT_AXIS_NORMAL, COMPAT_SIGNED_FRESNEL, COMPAT_ALL = 1, 2, 4, 7
NCOUNTERS = 16
COUNTER_NAMES = ["scatter", "boundary", "query", "roulette", "miss", "capped", "rz_drop",
                 "vox_drop", "photons", "draws", "safe_skip", "bvh_query", "bad_input", "bounds",
                 "region_mismatch", "agg_leaders"]
FIX_ONE = float(2 ** 32)

_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int32)
_up = C.POINTER(C.c_uint64)
_u32p = C.POINTER(C.c_uint32)


class Geometry(C.Structure):
    _fields_ = [(n, C.c_int32) for n in
                ("dimx", "dimy", "dimz", "dimR", "dimAlpha", "sft_nx", "sft_ny",
                 "rz_nr", "rz_nz", "kernel_dimR")]


class Tallies(C.Structure):
    _fields_ = [("sft", _up), ("rtd", _up), ("rz", _up), ("vox", _up), ("rbins", _up),
                ("region", _up), ("det", _up), ("counters", C.c_uint64 * NCOUNTERS),
                ("n_vox", C.c_int64), ("n_rbins", C.c_int64), ("n_region", C.c_int64),
                ("n_det", C.c_int64)]


class Stats(C.Structure):
    _fields_ = [("n_tri", C.c_int64), ("n_nodes", C.c_int64)] + \
        [(n, C.c_int32) for n in ("bvh_depth", "nodes_smem", "tris_smem", "smem_bytes", "blocks_per_sm",
                                  "grid", "block", "num_sms")] + \
        [("h2d_bytes", C.c_int64), ("d2h_bytes", C.c_int64), ("last_kernel_ms", C.c_float)]


class DeviceTallies(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in ("sft", "rtd", "rz", "vox", "rbins", "region", "det", "counters")] + \
        [(n, C.c_int64) for n in ("n_sft", "n_rtd", "n_rz", "n_vox", "n_rbins", "n_region", "n_det",
                                  "n_counters")] + [("stream", C.c_void_p), ("grad", C.c_void_p),
                                                    ("n_grad", C.c_int64)]


class NoAllocArgs(C.Structure):
    """lp_noalloc_args: mesh as device pointers, media on the host, outputs on the device."""
    _fields_ = [("tri", C.c_void_p), ("nrm", C.c_void_p), ("med", C.c_void_p), ("n_tri", C.c_int64),
                ("nmuasg", _fp), ("n_media", C.c_int32),
                ("p_start", C.c_float * 3), ("v_start", C.c_float * 3), ("ep0xyz", C.c_float * 12),
                ("fiber_radius", C.c_float), ("fiber_cos_max", C.c_float),
                ("dimensions", C.c_float * 3), ("det_grid", C.c_float * 6), ("fetal_id", C.c_int32),
                ("chance", C.c_float), ("w_threshold", C.c_float), ("factor", C.c_float),
                ("seed", C.c_uint64), ("compat", C.c_uint32), ("first", C.c_int64), ("n_photons", C.c_int64),
                ("sft", C.c_void_p), ("rtd", C.c_void_p), ("rz", C.c_void_p), ("region", C.c_void_p),
                ("counters", C.c_void_p)]


NOALLOC_MAX_TRI, NOALLOC_MAX_MEDIA = 4096, 64
GRAD_MAX_REGIONS = 8
BATCH_MAX_MEDIA = 8

_dp = C.POINTER(C.c_double)


class Instance(C.Structure):
    """lp_instance: one transport problem of a batch."""
    _fields_ = [("context", C.c_int32), ("n_media", C.c_int32), ("nmuasg", C.c_float * (4 * BATCH_MAX_MEDIA)),
                ("first", C.c_int64), ("n_photons", C.c_int64)]


class Gradient(C.Structure):
    """lp_gradient: ring signals and their derivatives (arrays owned by the context)."""
    _fields_ = [("n_det", C.c_int32), ("n_media", C.c_int32), ("n_photons", C.c_int64)] + \
        [(n, _dp) for n in ("signal", "signal_se", "d_mua", "d_mus", "d_mua_se", "d_mus_se")]


class LPError(RuntimeError):
    """Raised when a liblpcuda call returns a non-zero status."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"liblpcuda error {code} ({ERRORS.get(code, '?')}): {msg}")
        self.code = code


_lib = None

_SIGS = {
    "lp_create": ([C.POINTER(C.c_void_p), C.c_int], C.c_int),
    "lp_destroy": ([C.c_void_p], None),
    "lp_last_error": ([C.c_void_p], C.c_char_p),
    "lp_set_mesh": ([C.c_void_p, C.c_int64, _fp, _fp, _ip], C.c_int),
    "lp_set_media": ([C.c_void_p, C.c_int32, _fp], C.c_int),
    "lp_set_source": ([C.c_void_p, _fp, _fp, _ip, C.c_int32, _fp], C.c_int),
    "lp_set_tally_grid": ([C.c_void_p, _fp, _fp, C.c_int32], C.c_int),
    "lp_set_fiber_source": ([C.c_void_p, C.c_float, C.c_float], C.c_int),
    "lp_set_params": ([C.c_void_p, C.c_float, C.c_float, C.c_float, C.c_uint64, C.c_uint32], C.c_int),
    "lp_set_extra_tallies": ([C.c_void_p, _ip, _fp, C.c_int32, C.c_float, C.c_int32, _fp], C.c_int),
    "lp_set_max_steps": ([C.c_void_p, C.c_int64], C.c_int),
    "lp_set_arithmetic": ([C.c_void_p, C.c_int], C.c_int),
    "lp_set_safety_grid": ([C.c_void_p, C.c_int64], C.c_int),
    "lp_set_cell_lists": ([C.c_void_p, C.c_int], C.c_int),
    "lp_set_cell_margin": ([C.c_void_p, C.c_float], C.c_int),
    "lp_set_tally_aggregation": ([C.c_void_p, C.c_int], C.c_int),
    "lp_set_smem_budget": ([C.c_void_p, C.c_int32], C.c_int),
    "lp_set_exit_records": ([C.c_void_p, C.c_int64], C.c_int),
    "lp_run": ([C.c_void_p, C.c_int64, C.c_int64], C.c_int),
    "lp_run_async": ([C.c_void_p, C.c_int64, C.c_int64], C.c_int),
    "lp_sync": ([C.c_void_p], C.c_int),
    "lp_zero_tallies": ([C.c_void_p], C.c_int),
    "lp_get_geometry": ([C.c_void_p, C.POINTER(Geometry)], C.c_int),
    "lp_get_tallies": ([C.c_void_p, C.POINTER(Tallies)], C.c_int),
    "lp_set_tallies": ([C.c_void_p, C.POINTER(Tallies)], C.c_int),
    "lp_get_gradient_sums": ([C.c_void_p, C.POINTER(C.c_double), C.c_int64], C.c_int),
    "lp_set_gradient_sums": ([C.c_void_p, C.POINTER(C.c_double), C.c_int64], C.c_int),
    "lp_get_exit_records": ([C.c_void_p, _fp, C.c_int64], C.c_int),
    "lp_last_kernel_ms": ([C.c_void_p, _fp], C.c_int),
    "lp_query_triangles": ([C.c_void_p, C.c_int64, _fp, _fp, _ip, _fp, _ip, _fp], C.c_int),
    "lp_philox_blocks": ([C.c_int, _u32p, _u32p, C.c_int64, _u32p], C.c_int),
    "lp_get_stats": ([C.c_void_p, C.POINTER(Stats)], C.c_int),
    "lp_get_device_tallies": ([C.c_void_p, C.POINTER(DeviceTallies)], C.c_int),
    "lp_fp32_peak": ([C.c_int, C.POINTER(C.c_double)], C.c_int),
    "lp_l2_atomic_peak": ([C.c_int, C.POINTER(C.c_double)], C.c_int),
    "lp_debug_fail_allocation": ([C.c_int64], C.c_int),
    "lp_run_noalloc": ([C.POINTER(NoAllocArgs), C.c_void_p], C.c_int),
    "lp_batch_config_count": ([], C.c_int),
    "lp_batch_config_info": ([C.c_int32, _ip, _ip, _ip], C.c_int),
    "lp_batch_create": ([C.POINTER(C.c_void_p), C.c_int32, C.POINTER(C.c_void_p)], C.c_int),
    "lp_batch_destroy": ([C.c_void_p], None),
    "lp_batch_last_error": ([C.c_void_p], C.c_char_p),
    "lp_batch_set_instances": ([C.c_void_p, C.c_int32, C.POINTER(Instance)], C.c_int),
    "lp_batch_set_gradient": ([C.c_void_p, C.c_int], C.c_int),
    "lp_batch_set_plain_threshold": ([C.c_void_p, C.c_int64], C.c_int),
    "lp_batch_plain_count": ([C.c_void_p, C.POINTER(C.c_int32)], C.c_int),
    "lp_batch_set_config": ([C.c_void_p, C.c_int32], C.c_int),
    "lp_batch_autotune": ([C.c_void_p, C.c_int64, _ip, _dp], C.c_int),
    "lp_batch_run": ([C.c_void_p], C.c_int),
    "lp_batch_last_ms": ([C.c_void_p, _fp], C.c_int),
    "lp_batch_ring_signals": ([C.c_void_p, _dp, _dp], C.c_int),
    "lp_batch_get_tallies": ([C.c_void_p, C.c_int32, C.POINTER(Tallies)], C.c_int),
    "lp_batch_get_gradient": ([C.c_void_p, C.c_int32, C.POINTER(Gradient)], C.c_int),
    "lp_set_gradient": ([C.c_void_p, C.c_int], C.c_int),
    "lp_get_gradient": ([C.c_void_p, C.POINTER(Gradient)], C.c_int),
    "lp_forward": ([C.c_void_p, C.c_int64, C.c_int64, _dp], C.c_int),
    "lp_backward": ([C.c_void_p, _dp, _dp, _dp], C.c_int),
}

EXPORTED = sorted(_SIGS)


DEBUG_LIB_PATH = os.path.join(os.path.dirname(LIB_PATH), "liblpcuda_debug.so")


def lib():
    """Load liblpcuda.so (or, with LP_DEBUG_LIBRARY=1 in the environment, the bounds-checked
    build liblpcuda_debug.so); raises if it has not been built."""
    global _lib
    if _lib is None:
        path = DEBUG_LIB_PATH if os.environ.get("LP_DEBUG_LIBRARY") == "1" else LIB_PATH
        if not os.path.isfile(path):
            raise RuntimeError(f"{path} is missing: build it with lightpropagation_b200.build.build()")
        L = C.CDLL(path)
        for name, (args, res) in _SIGS.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _lib = L
    return _lib


def check(rc: int, ctx=None) -> None:
    if rc != LP_OK:
        msg = lib().lp_last_error(ctx)
        raise LPError(rc, msg.decode() if msg else "")


def check_batch(rc: int, batch=None) -> None:
    if rc != LP_OK:
        msg = lib().lp_batch_last_error(batch)
        raise LPError(rc, msg.decode() if msg else "")


def fptr(a):
    return a.ctypes.data_as(_fp)


def iptr(a):
    return a.ctypes.data_as(_ip)


def u32ptr(a):
    return a.ctypes.data_as(_u32p)
