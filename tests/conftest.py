import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import pyoracle as po  # noqa: E402


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and liblpcuda.so")


def to_case(w) -> "po.Case":
    """Workload (lightpropagation_b200.workloads) -> oracle Case."""
    return po.Case(tri=w.tri, nrm=w.nrm, med=w.med, nmuasg=w.nmuasg, p_start=w.p_start,
                   v_start=w.v_start, ep0xyz=w.ep0xyz, dimensions=w.dimensions,
                   det_grid=w.det_grid, fetal_id=w.fetal_id, chance=w.chance,
                   w_threshold=w.w_threshold, factor=w.factor, vox_n=w.vox_n, vox_d=w.vox_d,
                   n_rbins=w.n_rbins, rbin_dr=w.rbin_dr, det_r=w.det_r,
                   src_type=1 if (w.fiber_radius > 0 or w.fiber_na > 0) else 0,
                   src_radius=w.fiber_radius, src_cos_max=w.src_cos_max)


@pytest.fixture(scope="session")
def oracle_lib():
    po.build()
    return po.lib()


def z_scores(a_batches, b_batches):
    """Per-element z of the difference of two means from batch samples [B, ...]."""
    a = np.asarray(a_batches, np.float64)
    b = np.asarray(b_batches, np.float64)
    ma, mb = a.mean(0), b.mean(0)
    va = a.var(0, ddof=1) / a.shape[0]
    vb = b.var(0, ddof=1) / b.shape[0]
    se = np.sqrt(va + vb)
    with np.errstate(divide="ignore", invalid="ignore"):
        z = np.where(se > 0, (ma - mb) / se, np.where(ma == mb, 0.0, np.inf))
    return z
