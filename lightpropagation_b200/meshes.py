"""Synthetic triangle meshes and source geometry in the reference's layouts.

Meshes follow the conventions of the reference's OBJ import
(src/IO/ImportExport.cpp:952-1053): each triangle carries (inner, outer) region
ids, and its normal points from the inner region to the outer one (outward for a
closed object), so TransmitOrReflect (MCLightPropagation.cl:921-1018) enters the
outer region when the photon moves along the normal.
"""
from __future__ import annotations

import numpy as np

F = np.float32


def emitter_frame(heading):
    """Orthonormal basis with eZ = heading, in float32 as Emitter::CalculateEmitterModel
    computes it (src/Model/Emitter.cpp:311-339)."""
    ez = np.array(heading, F)
    if ez[2] != 0:
        a = np.array([1, 1, -(ez[0] + ez[1]) / ez[2]], F)
    elif ez[1] != 0:
        a = np.array([1, -ez[0] / ez[1], 0], F)
    else:
        a = np.array([0, 1, 0], F)

    def norm(v):
        f = F(np.sqrt(F(v[0] * v[0] + v[1] * v[1]) + F(v[2] * v[2])))
        return np.array([v[0] / f, v[1] / f, v[2] / f], F)

    def cross(a, b):
        return np.array([F(a[1] * b[2]) - F(a[2] * b[1]), F(a[2] * b[0]) - F(a[0] * b[2]),
                         F(a[0] * b[1]) - F(a[1] * b[0])], F)

    a = norm(a)
    ez = norm(ez)
    ey = norm(cross(ez, a))
    ex = norm(cross(ey, ez))
    return ex, ey, ez


def emitter_start(poi, heading, distance):
    """pStart = POI - heading * distance (Emitter::CalculatePointOfOrigin, Emitter.cpp:186-205)."""
    h = np.array(heading, F)
    p = np.array(poi, F)
    d = F(distance)
    return np.array([F(-h[i] * d) + p[i] for i in range(3)], F)


def face_normals(tri: np.ndarray) -> np.ndarray:
    """Unit normal (B - A) x (C - A) per triangle, computed in double."""
    t = tri.reshape(-1, 3, 3).astype(np.float64)
    n = np.cross(t[:, 1] - t[:, 0], t[:, 2] - t[:, 0])
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    return n.astype(F)


def _quad(p0, p1, p2, p3):
    """Two triangles of the planar quad p0-p1-p2-p3 (counter-clockwise seen from the normal side)."""
    return [p0 + p1 + p2, p0 + p2 + p3]


def layered_slab(thicknesses, half_width=50.0, z0=0.0):
    """Stacked boxes (one per layer) along +z with shared interfaces deduplicated.

    Region ids: 0 = ambient, layer k = k + 1.  Layer k's box has its top face only
    when k == 0 (the other tops coincide with the box above, whose bottom face
    carries inner = upper layer, outer = lower layer), four side faces (outer = 0)
    and a bottom face (outer = next layer or 0).  Returns tri [T,9], nrm [T,3],
    med [T,2] with 12 + 10 * (layers - 1) triangles.
    """
    w = float(half_width)
    tris, meds = [], []
    z = float(z0)
    n = len(thicknesses)
    for k, th in enumerate(thicknesses):
        zt, zb = z, z + float(th)
        inner = k + 1
        below = k + 2 if k + 1 < n else 0
        c = {  # corners: top (z = zt) and bottom (z = zb)
            "t00": [-w, -w, zt], "t10": [w, -w, zt], "t11": [w, w, zt], "t01": [-w, w, zt],
            "b00": [-w, -w, zb], "b10": [w, -w, zb], "b11": [w, w, zb], "b01": [-w, w, zb],
        }
        faces = []
        if k == 0:  # top face, normal -z (towards the ambient above)
            faces.append((_quad(c["t00"], c["t01"], c["t11"], c["t10"]), 0))
        faces.append((_quad(c["b00"], c["b10"], c["b11"], c["b01"]), below))       # bottom, +z
        faces.append((_quad(c["t00"], c["t10"], c["b10"], c["b00"]), 0))           # y = -w, -y
        faces.append((_quad(c["t01"], c["b01"], c["b11"], c["t11"]), 0))           # y = +w, +y
        faces.append((_quad(c["t00"], c["b00"], c["b01"], c["t01"]), 0))           # x = -w, -x
        faces.append((_quad(c["t10"], c["t11"], c["b11"], c["b10"]), 0))           # x = +w, +x
        for quad, outer in faces:
            for t in quad:
                tris.append(t)
                meds.append((inner, outer))
        z = zb
    tri = np.array(tris, F).reshape(-1, 9)
    return tri, face_normals(tri), np.array(meds, np.int32)
