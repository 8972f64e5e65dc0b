"""The mesh generators of the curved and deformed abdomen workloads, checked on the CPU.

The transport kernel trusts its mesh: every surface must be closed, its triangles must
carry the (inner, outer) region ids of the two sides, and the face normals must point
from inner to outer (the orientation the boundary code reads).  A surface that leaks or
two surfaces that cross would send photons into the wrong region without any error.
"""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

from lightpropagation_b200 import meshes  # noqa: E402


def shells(tri, freq):
    per = 20 * freq * freq
    assert tri.shape[0] % per == 0
    return [tri[k * per:(k + 1) * per].reshape(-1, 3, 3).astype(np.float64) for k in range(tri.shape[0] // per)]


def edge_counts(t):
    v = t.reshape(-1, 3)
    keys, inv = np.unique(v, axis=0, return_inverse=True)
    idx = inv.reshape(-1, 3)
    e = np.concatenate([idx[:, [0, 1]], idx[:, [1, 2]], idx[:, [2, 0]]])
    e.sort(axis=1)
    _, counts = np.unique(e, axis=0, return_counts=True)
    return counts


def signed_volume(t):
    return np.einsum("ij,ij->i", t[:, 0], np.cross(t[:, 1], t[:, 2])).sum() / 6.0


def inside_radially(inner_pts, outer_tri, margin):
    """Every inner point lies closer to the origin than the outer surface in its direction
    (the shells are star-shaped about the origin; the nearest sampled direction stands in)."""
    ov = np.unique(outer_tri.reshape(-1, 3), axis=0)
    orad = np.linalg.norm(ov, axis=1)
    odir = ov / orad[:, None]
    ip = inner_pts / np.linalg.norm(inner_pts, axis=1, keepdims=True)
    nearest = np.argmax(ip @ odir.T, axis=1)
    return np.all(np.linalg.norm(inner_pts, axis=1) + margin < orad[nearest])


@pytest.mark.parametrize("kind", ["curved", "deformed"])
def test_abdomen_surfaces_closed_oriented_and_nested(kind):
    freq = 16
    if kind == "curved":
        tri, nrm, med = meshes.curved_abdomen(freq=freq)
        expect = [(1, 0), (2, 1), (3, 2), (4, 3), (5, 4)]
    else:
        tri, nrm, med, pole = meshes.deformed_abdomen(freq=freq)
        expect = [(1, 0), (2, 1), (3, 2), (4, 3), (5, 4), (6, 4)]
        assert pole[2] < 0 and abs(pole[0]) < 1e-6 and abs(pole[1]) < 1e-6
    S = shells(tri, freq)
    assert len(S) == len(expect)
    per = 20 * freq * freq
    vols = []
    for k, t in enumerate(S):
        assert np.all(edge_counts(t) == 2), f"surface {k} is not closed"
        m = med[k * per:(k + 1) * per]
        assert np.all(m == np.array(expect[k])), f"surface {k} region ids"
        # outward normals <=> positive enclosed volume; the stored normals agree with the winding
        vols.append(signed_volume(t))
        assert vols[-1] > 0, f"surface {k} is wound inwards"
        fn = np.cross(t[:, 1] - t[:, 0], t[:, 2] - t[:, 0])
        assert np.all(np.einsum("ij,ij->i", fn, nrm[k * per:(k + 1) * per]) > 0)
    # the four maternal shells nest, and the head (and placenta) sit inside the fluid
    assert vols[0] > vols[1] > vols[2] > vols[3] > vols[4] > 0
    for k in range(3):
        assert inside_radially(S[k + 1].reshape(-1, 3), S[k], 0.5)
    assert inside_radially(S[4].reshape(-1, 3), S[3], 1.0), "fetal head crosses the uterine wall"
    if kind == "deformed":
        assert inside_radially(S[5].reshape(-1, 3), S[3], 1.0), "placenta crosses the uterine wall"


def test_workload_triangle_counts():
    assert 5 * 20 * 45 ** 2 == 202_500
    assert 6 * 20 * 129 ** 2 == 1_996_920
    tri, _, med = meshes.curved_abdomen(freq=45)
    assert tri.shape == (202_500, 9) and med.shape == (202_500, 2)


def test_batched_workload_spec():
    """The batched workload's draws follow its specification, its photon ranges tile one
    id range, and every head variant clears the uterine wall."""
    from lightpropagation_b200 import workloads
    spec = workloads.batched_abdomen(n_instances=64, freq=8, variant_freq=12)
    assert len(spec.meshes) == 9
    inst = spec.instances
    first = 0
    for i, d in enumerate(inst):
        assert d["mesh"] == i % 9
        assert d["wavelength"] == (660 if i % 2 == 0 else 940)
        assert 0.30 <= d["spo2_f"] <= 0.70 and 0.90 <= d["spo2_m"] <= 1.00
        assert 1e6 <= d["n_photons"] <= 1e8
        assert d["first"] == first
        first += d["n_photons"]
        nm = np.asarray(d["nmuasg"], np.float32).reshape(-1, 4)
        assert nm.shape[0] == 6 and np.all(nm[1:, 1] > 0) and np.all(nm[1:, 2] > 0)
    for w in spec.meshes[1:]:
        S = shells(np.asarray(w.tri), 12)
        assert inside_radially(S[4].reshape(-1, 3), S[3], 1.0), "a variant's head crosses the uterine wall"
