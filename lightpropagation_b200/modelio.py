"""Reference-format model loading through the C++ host layer (liblphost.so).

``load_model(config.xml)`` reads the <config> XML, the OBJ mesh and the emitter
file exactly as the C++ CalculatePropagation driver does (src/IO/ReadXML.cpp,
src/IO/ImportExport.cpp, src/Model/Emitter.cpp restated without VTK) and returns a
``workloads.Workload`` ready for ``Simulation``.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _native
from .workloads import Workload

HOST_LIB = os.path.join(os.path.dirname(os.path.abspath(__file__)), "liblphost.so")
LPSIM = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lpsim")
_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.isfile(HOST_LIB):
            raise RuntimeError(f"{HOST_LIB} is missing: build it with lightpropagation_b200.build.build()")
        _native.lib()  # liblpcuda.so first (liblphost.so links it)
        L = C.CDLL(HOST_LIB)
        L.lph_load.argtypes = [C.c_char_p, C.c_char_p, C.c_int]
        L.lph_load.restype = C.c_void_p
        L.lph_free.argtypes = [C.c_void_p]
        for name, rt in (("lph_tri", C.POINTER(C.c_float)), ("lph_nrm", C.POINTER(C.c_float)),
                         ("lph_vn", C.POINTER(C.c_float)), ("lph_med", C.POINTER(C.c_int32)),
                         ("lph_nmuasg", C.POINTER(C.c_float)), ("lph_n_tri", C.c_int64),
                         ("lph_n_media", C.c_int32)):
            f = getattr(L, name)
            f.argtypes = [C.c_void_p]
            f.restype = rt
        fp = C.POINTER(C.c_float)
        L.lph_source.argtypes = [C.c_void_p, fp, fp, fp]
        L.lph_grid.argtypes = [C.c_void_p, fp, fp, C.POINTER(C.c_int32), fp, fp, fp, C.POINTER(C.c_int64)]
        _lib = L
    return _lib


def load_model(config_path: str, n_photons: int = 0) -> Workload:
    L = lib()
    err = C.create_string_buffer(512)
    h = L.lph_load(config_path.encode(), err, 512)
    if not h:
        raise RuntimeError(f"load_model({config_path}): {err.value.decode()}")
    try:
        T = L.lph_n_tri(h)
        R = L.lph_n_media(h)
        arr = lambda p, n: np.ctypeslib.as_array(p, shape=(n,)).copy()
        tri = arr(L.lph_tri(h), 9 * T).reshape(T, 9)
        nrm = arr(L.lph_nrm(h), 3 * T).reshape(T, 3)
        vn = arr(L.lph_vn(h), 3 * T).reshape(T, 3)
        med = arr(L.lph_med(h), 2 * T).reshape(T, 2)
        nm = arr(L.lph_nmuasg(h), 4 * R).reshape(R, 4)
        p0, v0, ep = (np.zeros(3, np.float32), np.zeros(3, np.float32), np.zeros(12, np.float32))
        fp = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))
        L.lph_source(h, fp(p0), fp(v0), fp(ep))
        dims, dg = np.zeros(3, np.float32), np.zeros(6, np.float32)
        fetal, photons = C.c_int32(), C.c_int64()
        chance, wth, ppu = C.c_float(), C.c_float(), C.c_float()
        L.lph_grid(h, fp(dims), fp(dg), C.byref(fetal), C.byref(chance), C.byref(wth), C.byref(ppu),
                   C.byref(photons))
    finally:
        L.lph_free(h)
    w = Workload(name=os.path.basename(config_path), tri=tri, nrm=nrm, med=med, nmuasg=nm, p_start=p0,
                 v_start=v0, ep0xyz=ep, dimensions=dims, det_grid=dg, fetal_id=int(fetal.value),
                 n_photons=int(n_photons or photons.value), chance=float(chance.value),
                 w_threshold=float(wth.value), factor=float(ppu.value))
    w.file_normals = vn
    return w
