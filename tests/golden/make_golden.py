#!/usr/bin/env python3
"""Generate the golden fixtures under tests/golden/ from the reference itself.

Runs the reference kernel compiled for the CPU (oracle/_ref/libclref.so, built by
oracle/build_ref.py from src/Simulation/MCLightPropagation.cl and src/PSNR/PSNR.cpp)
on models shipped with the reference (models/model1, model2, model3 and the planar
5-region model4/modelPlanar.obj), one work-item at a time, with the ran3 table
seeded through PSNR::SetSeed.  Stores the kernel's inputs as passed (mesh arrays,
packed optical properties, source, grid), the per-photon float8 exit records, the
non-zero cells of the r-z buffer and the final RNG state.

Mesh arrays come from a minimal OBJ reading that follows
ImportExport::GenMediumIDsFromObjModel (src/IO/ImportExport.cpp:952-1053): region
ids from `o <name>` / `g <id>` / `g <id>_<surf>` lines, one triangle per `f` line,
per-face normal (B - A) x (C - A).  Only this script reads the reference checkout.

    python tests/golden/make_golden.py [--reference DIR] [case ...]   (DIR: $LP_REFERENCE_DIR)
"""
import argparse
import os
import re
import sys
import xml.etree.ElementTree as ET

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import pyoracle as po  # noqa: E402
from build_ref import reference_dir  # noqa: E402
from lightpropagation_b200 import meshes  # noqa: E402

CASES = [
    # name, model dir, obj, config, photons, ran3 seed
    ("model1", "model1", "model.obj", "config.xml", 2000, 1234),
    ("model2", "model2", "model.obj", "config.xml", 1500, 77),
    ("model3", "model3", "model.obj", "config.xml", 1500, 4242),
    ("model4_planar", "model4", "modelPlanar.obj", "configPlanar.xml", 600, 31),
    # the curved 5-region model (25,600 triangles); its mesh is stored as shared vertices
    # and faces, which arrays() expands
    ("model4_curved", "model4", "model.obj", "config.xml", 400, 8),
]


def arrays(z):
    """(tri [T, 9], nrm [T, 3], med [T, 2]) of a fixture: stored directly, or as shared
    vertices + faces with the per-face normals (B - A) x (C - A) recomputed."""
    if "tri" in z:
        return z["tri"], z["nrm"], z["med"]
    tri = z["verts"][z["faces"]].reshape(-1, 9).astype(np.float32)
    return tri, meshes.face_normals(tri), z["med"]


def read_config(path):
    root = ET.parse(path).getroot()
    tissues = []
    for t in root.iter("tissue"):
        def f(tag, default=0.0):
            e = t.find(tag)
            return float(e.text) if e is not None else default
        tissues.append((int(t.find("ID").text), t.find("name").text.strip(), f("refraction", 1.0),
                        f("mua"), f("mus"), f("anisotropy")))
    tissues.sort()
    model = root.find("model")
    dims = [float(model.find("dimensions").find(k).text) for k in ("x", "y", "z")]
    ppu = float(model.find("PixelPerUnit").text)
    em = root.find("Emittermodel")
    pos = [float(x.text) for x in list(em.find("position"))[:3]]
    head = [float(x.text) for x in list(em.find("heading"))[:3]]
    dist = float(em.find("distance").text)
    sp = root.find("SimulationParams")
    chance = float(sp.find("chance").text)
    wth = float(sp.find("weightThreshold").text)
    logs = root.find("Logs")
    grid = logs.find("DetectionGrid")
    det = [float(grid.find(k).text) for k in ("x", "y", "z", "r", "phi", "rho")]
    fetal = int(logs.find("fetalID").text)
    return dict(tissues=tissues, dims=dims, ppu=ppu, pos=pos, head=head, dist=dist,
                chance=chance, wth=wth, det=det, fetal=fetal)


def read_obj(path, names, indexed=False):
    verts, faces, med = [], [], []
    inner = outer = 0
    with open(path) as fh:
        for line in fh:
            line = line.rstrip("\n").rstrip("\r")
            if line.startswith("v "):
                verts.append([float(x) for x in line.split()[1:4]])
                continue
            m = re.fullmatch(r"o (\w+)", line)
            if m:
                for i, nm in enumerate(names):
                    if nm == m.group(1):
                        inner = i
                        break
                continue
            if re.fullmatch(r"f (.+)", line):
                idx = [int(tok.split("/")[0]) - 1 for tok in line.split()[1:]]
                faces.append(idx[:3])
                med.append((inner, outer))
                continue
            m = re.fullmatch(r"g (\d+)", line)
            if m:
                outer = int(m.group(1))
                continue
            m = re.fullmatch(r"g (\d+)_(\w+)", line)
            if m:
                outer = int(m.group(1))
    v = np.array(verts, np.float32)
    tri = np.stack([np.concatenate([v[a], v[b], v[c]]) for a, b, c in faces]).astype(np.float32)
    if indexed:
        return tri, meshes.face_normals(tri), np.array(med, np.int32), v, np.array(faces, np.int32)
    return tri, meshes.face_normals(tri), np.array(med, np.int32)


def make_case(ref_root, name, mdir, obj, cfg, n, seed):
    c = read_config(os.path.join(ref_root, "models", mdir, cfg))
    names = [t[1] for t in c["tissues"]]
    tri, nrm, med, verts, faces = read_obj(os.path.join(ref_root, "models", mdir, obj), names, indexed=True)
    nmuasg = np.array([[t[2], t[3], t[4], t[5]] for t in c["tissues"]], np.float32)
    ex, ey, ez = meshes.emitter_frame(c["head"])
    p0 = meshes.emitter_start(c["pos"], c["head"], c["dist"])
    ep = np.concatenate([np.array(c["pos"], np.float32), ex, ey, ez]).astype(np.float32)
    case = po.Case(tri=tri, nrm=nrm, med=med, nmuasg=nmuasg, p_start=p0,
                   v_start=np.array(c["head"], np.float32), ep0xyz=ep,
                   dimensions=np.array(c["dims"], np.float32), det_grid=np.array(c["det"], np.float32),
                   fetal_id=c["fetal"], chance=c["chance"], w_threshold=c["wth"], factor=c["ppu"])
    g = po.geometry(case)
    pad = 4 * g.rz_nr * g.rz_nz + 100000
    st0, ix0 = po.ref_ran3_state(seed)
    rec, rz, st, ix = po.ref_run(case, n, ran3_seed=seed, rz_pad=pad)
    cells = np.nonzero(np.any(rz != 0, axis=1))[0]
    mesh = dict(tri=tri, nrm=nrm, med=med) if tri.shape[0] < 1000 else dict(verts=verts, faces=faces, med=med)
    out = dict(**mesh, nmuasg=nmuasg, p_start=p0, v_start=case.v_start, ep0xyz=ep,
               dimensions=case.dimensions, det_grid=case.det_grid,
               emitter=np.array(c["pos"] + c["head"] + [c["dist"]], np.float32),
               tissue_names=np.array(names),
               scalars=np.array([c["fetal"], c["chance"], c["wth"], c["ppu"], n, seed, pad], np.float64),
               ran3_state0=st0, ran3_inext0=ix0, exit_rec=rec,
               rz_cells=(cells - pad).astype(np.int64), rz_vals=rz[cells], ran3_state1=st, ran3_inext1=ix)
    path = os.path.join(HERE, f"{name}.npz")
    np.savez_compressed(path, **out)
    print(f"{name}: {tri.shape[0]} triangles, {n} photons, {cells.size} r-z cells -> {path}")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=reference_dir())
    ap.add_argument("cases", nargs="*", help="names of the cases to make (default: all)")
    a = ap.parse_args()
    if not po.ref_available():
        import subprocess
        subprocess.check_call([sys.executable, os.path.join(ROOT, "oracle", "build_ref.py"),
                               "--reference", a.reference])
    po.build()
    for case in CASES:
        if not a.cases or case[0] in a.cases:
            make_case(a.reference, *case)


if __name__ == "__main__":
    main()
