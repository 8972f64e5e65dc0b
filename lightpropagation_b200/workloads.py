"""Named transport workloads (meshes, optical properties, source, tally layout).

``plain_slab`` is the small plain-method case: a 3-layer planar slab built as a
triangle mesh (skin 2 mm, fat 10 mm, uterus 30 mm; each layer a 100 x 100 mm box),
a normal-incidence pencil beam at the centre, 1e6 unit-weight photons, roulette
threshold 1e-4 with 1-in-10 survival, a 1 mm voxel absorption grid (100 x 100 x 42)
and 0.5 mm radial diffuse-reflectance bins.  Lengths are in mm and coefficients in
1/mm, so the reference's PixelPerUnit factor is 1.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import meshes

F = np.float32


@dataclass
class Workload:
    name: str
    tri: np.ndarray
    nrm: np.ndarray
    med: np.ndarray
    nmuasg: np.ndarray          # [R, 4] n, mua, mus, g
    p_start: np.ndarray
    v_start: np.ndarray
    ep0xyz: np.ndarray
    dimensions: np.ndarray
    det_grid: np.ndarray
    fetal_id: int
    n_photons: int
    chance: float = 0.1
    w_threshold: float = 1e-4
    factor: float = 1.0
    vox_n: tuple = (0, 0, 0)
    vox_d: tuple = (1.0, 1.0, 1.0)
    n_rbins: int = 0
    rbin_dr: float = 1.0
    det_r: Optional[np.ndarray] = None
    region_names: list = field(default_factory=list)

    @property
    def n_tri(self) -> int:
        return int(self.tri.shape[0])

    def apply(self, sim, seed=0x4C50, compat=7):
        """Load this workload into a propagation.Simulation."""
        sim.set_mesh(self.tri, self.nrm, self.med)
        sim.set_media(self.nmuasg)
        sim.set_source(self.p_start, self.v_start, self.ep0xyz)
        sim.set_tally_grid(self.dimensions, self.det_grid, self.fetal_id)
        sim.set_params(self.chance, self.w_threshold, self.factor, seed, compat)
        sim.set_extra_tallies(self.vox_n, self.vox_d, self.n_rbins, self.rbin_dr, self.det_r)
        return sim


def pencil_source(poi=(0.0, 0.0, 0.0), heading=(0.0, 0.0, 1.0), distance=1.0):
    ex, ey, ez = meshes.emitter_frame(heading)
    p0 = meshes.emitter_start(poi, heading, distance)
    ep = np.concatenate([np.array(poi, F), ex, ey, ez]).astype(F)
    return p0, np.array(heading, F), ep


def plain_slab(n_photons: int = 1_000_000) -> Workload:
    tri, nrm, med = meshes.layered_slab([2.0, 10.0, 30.0], half_width=50.0)
    nmuasg = np.array([[1.0, 0.0, 0.0, 0.0],      # ambient
                       [1.4, 0.02, 20.0, 0.9],    # skin
                       [1.44, 0.003, 12.0, 0.9],  # fat
                       [1.4, 0.02, 8.0, 0.9]],    # uterus / fetal tissue
                      F)
    p0, v0, ep = pencil_source()
    return Workload(
        name="plain_slab_3layer_32tri", tri=tri, nrm=nrm, med=med, nmuasg=nmuasg,
        p_start=p0, v_start=v0, ep0xyz=ep,
        dimensions=np.array([100.0, 100.0, 42.0], F),
        det_grid=np.array([1.0, 1.0, 1.0, 0.5, 1.0, 1.0], F),
        fetal_id=3, n_photons=n_photons,
        vox_n=(100, 100, 42), vox_d=(1.0, 1.0, 1.0), n_rbins=142, rbin_dr=0.5,
        region_names=["ambient", "skin", "fat", "uterus"])


WORKLOADS = {"plain_slab": plain_slab}
