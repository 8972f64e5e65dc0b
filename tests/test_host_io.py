"""C++ host layer (liblphost.so, lpsim) on the CPU: loaders and CLI without a GPU.

The reference's shipped models are read from the reference checkout when it is
present and compared with the kernel inputs stored in tests/golden/ (which the
reference kernel itself consumed); a synthetic model written in the same format
round-trips everywhere."""
import glob
import os
import subprocess

import numpy as np
import pytest

from build_ref import reference_dir
from golden.make_golden import arrays
from lightpropagation_b200 import meshes, modelio, workloads

REF = os.path.join(reference_dir(), "models")
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
CASES = {"model1": "model1/config.xml", "model2": "model2/config.xml", "model3": "model3/config.xml",
         "model4_planar": "model4/configPlanar.xml", "model4_curved": "model4/config.xml"}


@pytest.mark.skipif(not os.path.isdir(REF), reason="reference checkout not present")
@pytest.mark.parametrize("name", sorted(CASES))
def test_reference_models_load_as_the_kernel_saw_them(name):
    w = modelio.load_model(os.path.join(REF, CASES[name]))
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    tri, nrm, med = arrays(z)
    assert np.array_equal(w.tri.view(np.uint32), tri.view(np.uint32))
    assert np.array_equal(w.med, med)
    assert np.array_equal(w.nmuasg.view(np.uint32), z["nmuasg"].view(np.uint32))
    assert np.allclose(w.nrm, nrm, atol=1e-6)
    for k in ("p_start", "v_start", "ep0xyz", "dimensions", "det_grid"):
        assert np.array_equal(getattr(w, k).view(np.uint32), z[k].view(np.uint32)), k
    # the per-face normals agree with the vn records Blender wrote into the file
    has = np.linalg.norm(w.file_normals, axis=1) > 0
    assert np.allclose(w.nrm[has], w.file_normals[has], atol=1e-5)


def test_synthetic_model_round_trip(tmp_path):
    w = workloads.plain_slab()
    names = ["outside", "skin", "fat", "uterus"]
    meshes.write_obj(str(tmp_path / "slab.obj"), w.tri, w.med, names)
    (tmp_path / "emitter.txt").write_text("0 1\n")
    tissues = [(nm, *w.nmuasg[i]) for i, nm in enumerate(names)]
    meshes.write_config(str(tmp_path / "config.xml"), "/nonexistent/dir/slab.obj", tissues, w.dimensions,
                        w.det_grid, (0, 0, 0), (0, 0, 1), 1.0, 12345, w.fetal_id,
                        emitter_file="/nonexistent/dir/emitter.txt")
    m = modelio.load_model(str(tmp_path / "config.xml"))
    assert np.array_equal(m.tri.view(np.uint32), w.tri.view(np.uint32))
    assert np.array_equal(m.med, w.med)
    assert np.allclose(m.nrm, w.nrm, atol=1e-6)
    assert np.array_equal(m.nmuasg, w.nmuasg)
    assert np.array_equal(m.p_start.view(np.uint32), w.p_start.view(np.uint32))
    assert np.array_equal(m.ep0xyz.view(np.uint32), w.ep0xyz.view(np.uint32))
    assert m.n_photons == 12345 and m.fetal_id == w.fetal_id


def test_missing_model_is_reported(tmp_path):
    meshes.write_config(str(tmp_path / "c.xml"), "/no/such.obj", [("outside", 1, 0, 0, 0)], (1, 1, 1),
                        (1, 1, 1, 1, 1, 1), (0, 0, 0), (0, 0, 1), 1, 10, 1)
    with pytest.raises(RuntimeError, match="cannot open"):
        modelio.load_model(str(tmp_path / "c.xml"))


def test_lpsim_loads_without_simulating(tmp_path):
    w = workloads.plain_slab()
    names = ["outside", "skin", "fat", "uterus"]
    meshes.write_obj(str(tmp_path / "slab.obj"), w.tri, w.med, names)
    (tmp_path / "emitter.txt").write_text("0 1\n")
    meshes.write_config(str(tmp_path / "config.xml"), "slab.obj", [(nm, *w.nmuasg[i]) for i, nm in enumerate(names)],
                        w.dimensions, w.det_grid, (0, 0, 0), (0, 0, 1), 1.0, 100, 3)
    r = subprocess.run([modelio.LPSIM, "-f", str(tmp_path / "config.xml"), "-v"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert "32 triangles, 4 regions" in r.stdout
