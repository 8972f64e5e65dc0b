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


def geodesic_sphere(freq: int):
    """Unit sphere from an icosahedron whose faces are split into freq^2 triangles.

    Returns vertices [V,3] (float64, unit length) and faces [20*freq^2, 3] (int, counter-
    clockwise seen from outside).  Vertices on shared icosahedron edges are created once,
    so neighbouring triangles share bit-identical edge vertices."""
    t = (1.0 + 5 ** 0.5) / 2.0
    ico_v = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t],
                      [0, -1, -t], [0, 1, -t], [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], np.float64)
    ico_v /= np.linalg.norm(ico_v, axis=1, keepdims=True)
    ico_f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
             (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5),
             (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    n = int(freq)
    verts = [v for v in ico_v]
    key_to_id = {("c", i): i for i in range(12)}

    def vid(face, i, j):
        a, b, c = face
        k = n - i - j
        # canonical key: a corner, a point on an edge (by sorted endpoints), or a face-interior point
        if i == n:
            return key_to_id[("c", b)]
        if j == n:
            return key_to_id[("c", c)]
        if k == n:
            return key_to_id[("c", a)]
        if k == 0:
            e, s = (b, c), j
        elif i == 0:
            e, s = (a, c), j
        elif j == 0:
            e, s = (a, b), i
        else:
            e = None
        if e is not None:
            lo, hi = min(e), max(e)
            pos = s if e[0] == lo else n - s
            key = ("e", lo, hi, pos)
            if key not in key_to_id:
                p = ico_v[lo] * (n - pos) / n + ico_v[hi] * pos / n
                key_to_id[key] = len(verts)
                verts.append(p / np.linalg.norm(p))
            return key_to_id[key]
        key = ("f", face, i, j)
        if key not in key_to_id:
            p = ico_v[a] * k / n + ico_v[b] * i / n + ico_v[c] * j / n
            key_to_id[key] = len(verts)
            verts.append(p / np.linalg.norm(p))
        return key_to_id[key]

    faces = []
    for f in ico_f:
        for i in range(n):
            for j in range(n - i):
                faces.append((vid(f, i, j), vid(f, i + 1, j), vid(f, i, j + 1)))
                if i + j < n - 1:
                    faces.append((vid(f, i + 1, j), vid(f, i + 1, j + 1), vid(f, i, j + 1)))
    return np.array(verts, np.float64), np.array(faces, np.int64)


def smooth_noise(u: np.ndarray, seed: int, terms: int = 12, freq: float = 2.0) -> np.ndarray:
    """Seeded smooth scalar field on the unit sphere, scaled to [0, 1]."""
    rng = np.random.default_rng(seed)
    k = rng.normal(size=(terms, 3))
    k *= freq / np.linalg.norm(k, axis=1, keepdims=True)
    ph = rng.uniform(0, 2 * np.pi, terms)
    amp = rng.uniform(0.5, 1.0, terms)
    s = (amp[None, :] * np.cos(u @ k.T + ph[None, :])).sum(1)
    return (s - s.min()) / (s.max() - s.min())


def _shell_triangles(points: np.ndarray, faces: np.ndarray, inner: int, outer: int):
    tri = points[faces].reshape(-1, 9).astype(F)
    med = np.tile(np.array([[inner, outer]], np.int32), (faces.shape[0], 1))
    return tri, med


def curved_abdomen(freq: int = 45, axes=(150.0, 120.0, 100.0), skin=2.0, fat=(8.0, 15.0), uterus=10.0,
                   head_radius=45.0, head_depth=40.0, noise_seed=2):
    """Nested shells of a maternal ellipsoid plus a fetal head sphere.

    Regions: 0 ambient, 1 skin, 2 fat, 3 uterus, 4 amniotic fluid, 5 fetal head.
    The outer ellipsoid (semi-axes a, b, c) is offset inwards along its normal by the
    skin thickness, then by a fat thickness that varies smoothly in [fat[0], fat[1]]
    (seeded noise over the sphere), then by the uterus thickness; inside lies the
    amniotic fluid.  The head sphere sits on the -z axis below the source at z = -c,
    its nearest surface head_depth below the skin.  Every surface is a geodesic
    sphere of the given frequency (20 * freq^2 triangles), so freq = 45 gives
    5 x 40500 = 202,500 triangles.  Normals point outwards (inner -> outer region)."""
    a, b, c = axes
    u, faces = geodesic_sphere(freq)
    p0 = u * np.array([a, b, c])[None, :]
    nrm = p0 / np.array([a * a, b * b, c * c])[None, :]
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    t_fat = fat[0] + (fat[1] - fat[0]) * smooth_noise(u, noise_seed)
    depths = [np.zeros(len(u)), np.full(len(u), skin), skin + t_fat, skin + t_fat + uterus]
    regions = [(1, 0), (2, 1), (3, 2), (4, 3)]
    tris, meds = [], []
    for d, (inner, outer) in zip(depths, regions):
        pts = p0 - d[:, None] * nrm
        t, m = _shell_triangles(pts, faces, inner, outer)
        tris.append(t)
        meds.append(m)
    centre = np.array([0.0, 0.0, -c + head_depth + head_radius])
    t, m = _shell_triangles(centre[None, :] + head_radius * u, faces, 5, 4)
    tris.append(t)
    meds.append(m)
    tri = np.concatenate(tris)
    med = np.concatenate(meds)
    return tri, face_normals(tri), med


class GradientNoise:
    """Seeded 3-D gradient noise after Perlin's improved noise (SIGGRAPH 2002): a lattice
    with a shuffled permutation table, one of 12 edge gradients per lattice point, the
    quintic fade 6t^5 - 15t^4 + 10t^3 and trilinear blending.  Values lie in about [-1, 1]."""

    GRAD = np.array([[1, 1, 0], [-1, 1, 0], [1, -1, 0], [-1, -1, 0], [1, 0, 1], [-1, 0, 1], [1, 0, -1],
                     [-1, 0, -1], [0, 1, 1], [0, -1, 1], [0, 1, -1], [0, -1, -1]], np.float64)

    def __init__(self, seed: int):
        perm = np.random.default_rng(seed).permutation(256)
        self.p = np.concatenate([perm, perm]).astype(np.int64)

    def __call__(self, x: np.ndarray) -> np.ndarray:
        x = np.asarray(x, np.float64)
        i0 = np.floor(x).astype(np.int64)
        f = x - i0
        i0 &= 255
        w = f * f * f * (f * (f * 6.0 - 15.0) + 10.0)
        p = self.p
        out = 0.0
        for dx in (0, 1):
            for dy in (0, 1):
                for dz in (0, 1):
                    h = p[p[p[i0[:, 0] + dx] + i0[:, 1] + dy] + i0[:, 2] + dz] % 12
                    g = self.GRAD[h]
                    d = g[:, 0] * (f[:, 0] - dx) + g[:, 1] * (f[:, 1] - dy) + g[:, 2] * (f[:, 2] - dz)
                    wx = w[:, 0] if dx else 1.0 - w[:, 0]
                    wy = w[:, 1] if dy else 1.0 - w[:, 1]
                    wz = w[:, 2] if dz else 1.0 - w[:, 2]
                    out = out + wx * wy * wz * d
        return out


def octave_noise(points: np.ndarray, seed: int, octaves: int = 3, scale: float = 40.0) -> np.ndarray:
    """Sum of `octaves` octaves of gradient noise (frequency x2, amplitude /2 each) at
    points [N, 3] (mm), with a feature size of `scale` mm, divided by the sum of the
    octave amplitudes (a fixed field: the value at a point does not depend on the others)."""
    noise = GradientNoise(seed)
    s = np.zeros(points.shape[0])
    amp, tot = 1.0, 0.0
    for o in range(octaves):
        s += amp * noise(points * (2.0 ** o) / scale + 17.31 * o)
        tot += amp
        amp *= 0.5
    return np.clip(s / tot, -1.0, 1.0)


def deformed_abdomen(freq: int = 129, axes=(150.0, 120.0, 100.0), skin=2.0, fat=(8.0, 15.0), uterus=10.0,
                     head_radius=45.0, head_depth=40.0, placenta_center=(0.0, 0.0, 52.0),
                     placenta_axes=(45.0, 45.0, 8.0), amplitude=3.0, seed=5):
    """The abdomen of `curved_abdomen` with a placenta and seeded 3-octave gradient-noise
    displacement of every surface (amplitude `amplitude` mm along the surface normal).

    Regions: 0 ambient, 1 skin, 2 fat, 3 uterus, 4 amniotic fluid, 5 fetal head,
    6 placenta (an ellipsoid in the amniotic fluid on the uterine wall opposite the
    source).  The four nested shells share one displacement field, so every layer keeps
    its thickness; the head and placenta get their own fields.  Six geodesic surfaces of
    20 * freq^2 triangles: freq 129 gives 1,996,920 triangles.  Returns (tri, nrm, med,
    pole): pole is the displaced outer-surface point on the -z axis (the source site)."""
    a, b, c = axes
    u, faces = geodesic_sphere(freq)
    p0 = u * np.array([a, b, c])[None, :]
    nrm = p0 / np.array([a * a, b * b, c * c])[None, :]
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    disp = amplitude * octave_noise(p0, seed)
    t_fat = fat[0] + (fat[1] - fat[0]) * smooth_noise(u, 2)
    depths = [np.zeros(len(u)), np.full(len(u), skin), skin + t_fat, skin + t_fat + uterus]
    regions = [(1, 0), (2, 1), (3, 2), (4, 3)]
    tris, meds = [], []
    for d, (inner, outer) in zip(depths, regions):
        pts = p0 + (disp - d)[:, None] * nrm
        t, m = _shell_triangles(pts, faces, inner, outer)
        tris.append(t)
        meds.append(m)
    centre = np.array([0.0, 0.0, -c + head_depth + head_radius])
    head = centre[None, :] + (head_radius + amplitude * octave_noise(u * head_radius, seed + 1))[:, None] * u
    t, m = _shell_triangles(head, faces, 5, 4)
    tris.append(t)
    meds.append(m)
    pc = np.array(placenta_center)[None, :]
    pl = pc + u * np.array(placenta_axes)[None, :]
    pn = u / np.array(placenta_axes)[None, :]
    pn /= np.linalg.norm(pn, axis=1, keepdims=True)
    pl = pl + (amplitude * octave_noise(pl, seed + 2))[:, None] * pn * 0.5
    t, m = _shell_triangles(pl, faces, 6, 4)
    tris.append(t)
    meds.append(m)
    tri = np.concatenate(tris)
    med = np.concatenate(meds)
    # the outer surface on the -z axis, where the normal is -z
    pole = np.array([0.0, 0.0, -c - amplitude * octave_noise(np.array([[0.0, 0.0, -c]]), seed)[0]], F)
    return tri, face_normals(tri), med, pole


def write_obj(path, tri: np.ndarray, med: np.ndarray, names) -> None:
    """Write a mesh in the reference's OBJ convention (ImportExport.cpp:952-1053):
    runs of triangles with the same (inner, outer) pair become `o <names[inner]>`,
    `g <outer>` and one `f` line per triangle (vertex order kept, so normals keep
    their orientation).  Vertices are written with 9 significant digits, which
    round-trips float32 exactly."""
    tri = np.asarray(tri, F).reshape(-1, 9)
    med = np.asarray(med, np.int32).reshape(-1, 2)
    with open(path, "w") as f:
        f.write("# written by lightpropagation_b200.meshes.write_obj\n")
        for v in tri.reshape(-1, 3):
            f.write("v %.9g %.9g %.9g\n" % (v[0], v[1], v[2]))
        last = None
        for i, (inner, outer) in enumerate(med):
            if last is None or inner != last[0]:
                f.write(f"o {names[inner]}\n")
                last = None
            if last is None or outer != last[1]:
                f.write(f"g {outer}\n")
            f.write(f"f {3 * i + 1} {3 * i + 2} {3 * i + 3}\n")
            last = (inner, outer)


def write_config(path, model_file, tissues, dims, det_grid, emitter_pos, emitter_heading, distance,
                 photons, fetal_id, chance=0.1, w_threshold=1e-4, ppu=1.0, emitter_file="emitter.txt"):
    """Write a <config> XML with the keys ReadXML reads (src/IO/ReadXML.cpp:109-870).
    tissues: list of (name, n, mua, mus, g) in region order."""
    t = "\n".join(
        f"      <tissue><ID>{i}</ID><name>{nm}</name><anisotropy>{g}</anisotropy><mua>{mua}</mua>"
        f"<mus>{mus}</mus><refraction>{n}</refraction></tissue>" for i, (nm, n, mua, mus, g) in enumerate(tissues))
    xyz = lambda v: "".join(f"<{k}>{x}</{k}>" for k, x in zip("xyz", v))
    g = "".join(f"<{k}>{x}</{k}>" for k, x in zip(("x", "y", "z", "r", "phi", "rho"), det_grid))
    with open(path, "w") as f:
        f.write(f"""<?xml version='1.0' encoding="utf-8"?>
<config>
  <model>
    <modelfile>{model_file}</modelfile>
    <unit>mm</unit>
    <PixelPerUnit>{ppu}</PixelPerUnit>
    <dimensions>{xyz(dims)}</dimensions>
    <tissueList>
{t}
    </tissueList>
  </model>
  <Emittermodel>
    <file>{emitter_file}</file>
    <position>{xyz(emitter_pos)}</position>
    <distance>{distance}</distance>
    <heading>{xyz(emitter_heading)}</heading>
  </Emittermodel>
  <SimulationParams>
    <numberOfPhotons>{photons}</numberOfPhotons>
    <chance>{chance}</chance>
    <weightThreshold>{w_threshold}</weightThreshold>
  </SimulationParams>
  <Logs>
    <fetalID>{fetal_id}</fetalID>
    <DetectionGrid>{g}</DetectionGrid>
  </Logs>
</config>
""")


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
