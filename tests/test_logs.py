"""Reference-format outputs of the C++ host layer (lp::Logs, lp::Analysis in liblphost.so)
on the CPU: each writer's file is parsed back and compared with the reference's
formulas restated in numpy -- layouts of Logs::SaveSurfaceArr / SaveRecordRd
(src/IO/Logs.cpp:337-402), the scale factors Scale2D, ScalePerRadius1D, ScalePerAngle1D
(Logs.cpp:493-516, 651-672), the per-radius / per-angle profiles (Logs.cpp:521-561,
674-713), FluenceZ (Logs.cpp:1075-1110) and the surface sums of Analysis
(Analysis.cpp:144-156, 447-463).  The files hold 6 significant digits (the default
stream precision, as in the reference), so they are compared to 1e-5 relative."""
import ctypes as C
import math

import numpy as np
import pytest

from lightpropagation_b200 import modelio

GRID = np.array([1.0, 1.0, 2.0, 0.5, 1.0, 1.5], np.float32)   # dx dy dz dr phi rho
N = 250000


def _lib():
    L = modelio.lib()
    L.lph_write_log.argtypes = [C.c_char_p, C.c_char_p, C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_int32),
                                C.c_int, C.POINTER(C.c_float), C.c_int64]
    L.lph_write_log.restype = C.c_int
    L.lph_surface_sums.argtypes = [C.POINTER(C.c_float), C.POINTER(C.c_int32), C.POINTER(C.c_double)]
    return L


def _write(tmp_path, kind, img, ext, fname="img.txt"):
    L = _lib()
    ncomp = img.shape[-1]
    v = np.ascontiguousarray(img, np.float32)
    e = np.array(ext, np.int32)
    rc = L.lph_write_log((str(tmp_path) + "/").encode(), fname.encode(), kind, v.ctypes.data_as(C.POINTER(C.c_float)),
                         e.ctypes.data_as(C.POINTER(C.c_int32)), ncomp, GRID.ctypes.data_as(C.POINTER(C.c_float)), N)
    assert rc == 0


def _read(path):
    return [[float(x) for x in line.split("\t") if x.strip()] for line in open(path) if line.strip()]


def scale2d(ir, ia):
    dr, da = float(GRID[3]), float(GRID[5]) * math.pi / 180
    s1 = np.float32(4.0 * math.pi * math.pi * dr * math.sin(da / 2) * dr * N)
    return np.float32(1.0 / ((ir + 0.5) * math.sin(2.0 * (ia + 0.5) * da) * float(s1)))


def per_radius(ir):
    dr = float(GRID[3])
    s1 = np.float32(2.0 * math.pi * dr * dr * N)
    return np.float32(1.0 / ((ir + 0.5) * float(s1)))


def per_angle(ia):
    da = float(GRID[5]) * math.pi / 180
    s1 = np.float32(2.0 * math.pi * da * N)
    return np.float32(1.0 / (math.sin((ia + 0.5) * da) * float(s1)))


@pytest.fixture(scope="module")
def images():
    rng = np.random.default_rng(3)
    sft = rng.uniform(0, 5, (7, 9, 3)).astype(np.float32)      # y in [-3, 3], x in [-4, 4]
    rtd = rng.uniform(0, 5, (6, 8, 1)).astype(np.float32)      # alpha in [0, 5], r in [0, 7]
    rz = rng.uniform(0, 5, (5, 11, 1)).astype(np.float32)      # z in [-4, 0], r in [-5, 5]
    return sft, rtd, rz


def test_surface_array_layout(tmp_path, images):
    sft, _, _ = images
    _write(tmp_path, 0, sft, (-4, 4, -3, 3, 0, 0), "surf.txt")
    rows = _read(tmp_path / "surf.txt")
    assert np.allclose(np.array(rows), sft[:, :, 0], rtol=1e-5)


def test_record_rd_scaled(tmp_path, images):
    _, rtd, _ = images
    _write(tmp_path, 1, rtd, (0, 7, 0, 5, 0, 0), "rtd.txt")
    got = np.array(_read(tmp_path / "rtd_Rd.txt"))
    want = np.array([[rtd[a, r, 0] * scale2d(r, a) for r in range(8)] for a in range(6)])
    assert np.allclose(got, want, rtol=1e-5)


def test_reflectance_per_radius_and_angle(tmp_path, images):
    _, rtd, _ = images
    _write(tmp_path, 2, rtd, (0, 7, 0, 5, 0, 0), "rtd.txt")
    _write(tmp_path, 3, rtd, (0, 7, 0, 5, 0, 0), "rtd.txt")
    pr = np.array(_read(tmp_path / "rtd_perRadius.txt"))
    pa = np.array(_read(tmp_path / "rtd_perAngle.txt"))
    assert np.allclose(pr[:, 0], np.arange(8) * GRID[3])
    assert np.allclose(pr[:, 1], [rtd[:, r, 0].sum(dtype=np.float32) * per_radius(r) for r in range(8)], rtol=1e-5)
    assert np.allclose(pa[:, 0], np.arange(6) * GRID[5])
    assert np.allclose(pa[:, 1], [rtd[a, :, 0].sum(dtype=np.float32) * per_angle(a) for a in range(6)], rtol=1e-5)


def test_fluence_per_depth(tmp_path, images):
    _, _, rz = images
    _write(tmp_path, 4, rz, (-5, 5, -4, 0, 0, 0), "phirz.txt")
    got = np.array(_read(tmp_path / "phirz_perZ.txt"))
    zs = np.arange(-4, 1)
    assert np.allclose(got[:, 0], np.abs(zs) * GRID[2])
    want = [rz[z + 4, :, 0].sum(dtype=np.float32) / np.float32(GRID[2] * N) for z in zs]
    assert np.allclose(got[:, 1], want, rtol=1e-5)


def test_analysis_surface_sums(images):
    sft, _, _ = images
    L = _lib()
    out = np.zeros(3)
    v = np.ascontiguousarray(sft, np.float32)
    e = np.array((-4, 4, -3, 3, 0, 0), np.int32)
    L.lph_surface_sums(v.ctypes.data_as(C.POINTER(C.c_float)), e.ctypes.data_as(C.POINTER(C.c_int32)),
                       out.ctypes.data_as(C.POINTER(C.c_double)))
    # Analysis accumulates in float, x outer and y inner (Analysis.cpp:447-463)
    want = []
    for c in range(3):
        s = np.float32(0)
        for x in range(9):
            for y in range(7):
                s = np.float32(s + sft[y, x, c])
        want.append(float(s))
    assert out[0] == want[0] and out[1] == want[1] and out[2] == want[2]
