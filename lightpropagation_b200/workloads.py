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
    fiber_radius: float = 0.0
    fiber_na: float = 0.0
    # reference behaviours kept (LP_COMPAT_*): 7 keeps all of them (the reference's own
    # pencil-beam layouts); 0 uses the corrected physics, needed wherever light enters a
    # region obliquely against a face normal (the signed-cosine Fresnel of the
    # reference reflects every such photon)
    compat: int = 7

    @property
    def n_tri(self) -> int:
        return int(self.tri.shape[0])

    @property
    def src_cos_max(self) -> float:
        """cos of the fibre cone half-angle, in float32 as the library computes it."""
        s = np.float32(self.fiber_na) / np.float32(self.nmuasg[0, 0])
        return float(np.sqrt(np.float32(1.0) - s * s))

    def apply(self, sim, seed=0x4C50, compat=None):
        """Load this workload into a propagation.Simulation."""
        compat = self.compat if compat is None else compat
        sim.set_mesh(self.tri, self.nrm, self.med)
        sim.set_media(self.nmuasg)
        sim.set_source(self.p_start, self.v_start, self.ep0xyz)
        sim.set_tally_grid(self.dimensions, self.det_grid, self.fetal_id)
        sim.set_params(self.chance, self.w_threshold, self.factor, seed, compat)
        sim.set_extra_tallies(self.vox_n, self.vox_d, self.n_rbins, self.rbin_dr, self.det_r)
        sim.set_fiber_source(self.fiber_radius, self.fiber_na)
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


# Optical properties of the abdomen regions (n, mua [1/mm], mus [1/mm], g) at the two
# wavelengths.  Synthetic values in the usual literature ranges for skin, fat, uterine
# wall and fetal head; the amniotic fluid values are the benchmark's own.  They are
# inputs of the benchmark, not measurements.
ABDOMEN_MEDIA = {
    660: [[1.0, 0.0, 0.0, 0.0],        # ambient
          [1.4, 0.02, 20.0, 0.9],      # skin
          [1.44, 0.003, 12.0, 0.9],    # fat
          [1.4, 0.02, 8.0, 0.9],       # uterus
          [1.33, 0.001, 0.1, 0.9],     # amniotic fluid
          [1.4, 0.015, 10.0, 0.9]],    # fetal head
    940: [[1.0, 0.0, 0.0, 0.0],
          [1.4, 0.015, 15.0, 0.9],
          [1.44, 0.004, 10.0, 0.9],
          [1.4, 0.025, 7.0, 0.9],
          [1.33, 0.001, 0.1, 0.9],
          [1.4, 0.02, 8.0, 0.9]],
}
RING_SEPARATIONS_MM = (20.0, 36.0, 52.0, 68.0, 84.0, 100.0)


def curved_abdomen(n_photons: int = 10_000_000, wavelength: int = 660, freq: int = 45, head_depth: float = 40.0,
                   fat=(8.0, 15.0)) -> Workload:
    """Curved mesh abdomen: maternal ellipsoid (semi-axes 150/120/100 mm) with nested
    skin (2 mm), fat (8-15 mm, seeded smooth noise), uterus (10 mm) shells, amniotic
    fluid inside, and a fetal head sphere (radius 45 mm, nearest surface 40 mm below the
    skin); 5 x 20 * freq^2 triangles (202,500 at freq 45).  A 0.4 mm NA-0.22 fibre at the
    -z pole points into the body; six 1 mm wide ring detectors at 20-100 mm.
    head_depth and fat give the variants of the batched workload; the source, tally
    layout and outer surface stay the same."""
    tri, nrm, med = meshes.curved_abdomen(freq=freq, head_depth=head_depth, fat=tuple(fat))
    nmuasg = np.array(ABDOMEN_MEDIA[int(wavelength)], F)
    p0, v0, ep = pencil_source(poi=(0.0, 0.0, -100.0), heading=(0.0, 0.0, 1.0), distance=1.0)
    det_r = np.array([[r - 0.5, r + 0.5] for r in RING_SEPARATIONS_MM], F)
    return Workload(
        name=f"curved_abdomen_{wavelength}nm_{tri.shape[0]}tri" +
             ("" if (head_depth, tuple(fat)) == (40.0, (8.0, 15.0)) else f"_head{head_depth:g}_fat{fat[0]:g}-{fat[1]:g}"),
        tri=tri, nrm=nrm, med=med, nmuasg=nmuasg,
        p_start=p0, v_start=v0, ep0xyz=ep,
        dimensions=np.array([300.0, 240.0, 200.0], F),
        det_grid=np.array([1.0, 1.0, 1.0, 0.5, 1.0, 1.0], F),
        fetal_id=5, n_photons=n_photons,
        vox_n=(200, 200, 120), vox_d=(1.0, 1.0, 1.0), n_rbins=300, rbin_dr=0.5, det_r=det_r,
        region_names=["ambient", "skin", "fat", "uterus", "amniotic", "fetal_head"],
        fiber_radius=0.2, fiber_na=0.22, compat=0)


PLACENTA = [1.4, 0.05, 10.0, 0.9]


def deformed_abdomen(n_photons: int = 10_000_000, wavelength: int = 660, freq: int = 129,
                     amplitude: float = 3.0, seed: int = 5, head_depth: float = 40.0) -> Workload:
    """The large deformed abdomen: the curved abdomen's shells plus a placenta (mua 0.05,
    mus 10 /mm), every surface displaced by seeded 3-octave gradient noise of amplitude
    3 mm; 7 regions and 6 x 20 * freq^2 triangles (1,996,920 at freq 129).  Same fibre
    source (at the displaced pole), rings and tally layout as curved_abdomen."""
    tri, nrm, med, pole = meshes.deformed_abdomen(freq=freq, amplitude=amplitude, seed=seed, head_depth=head_depth)
    nmuasg = np.array(ABDOMEN_MEDIA[int(wavelength)] + [PLACENTA], F)
    p0, v0, ep = pencil_source(poi=tuple(float(x) for x in pole), heading=(0.0, 0.0, 1.0), distance=1.0)
    det_r = np.array([[r - 0.5, r + 0.5] for r in RING_SEPARATIONS_MM], F)
    return Workload(
        name=f"deformed_abdomen_{wavelength}nm_{tri.shape[0]}tri", tri=tri, nrm=nrm, med=med, nmuasg=nmuasg,
        p_start=p0, v_start=v0, ep0xyz=ep,
        dimensions=np.array([300.0, 240.0, 200.0], F),
        det_grid=np.array([1.0, 1.0, 1.0, 0.5, 1.0, 1.0], F),
        fetal_id=5, n_photons=n_photons,
        vox_n=(200, 200, 120), vox_d=(1.0, 1.0, 1.0), n_rbins=300, rbin_dr=0.5, det_r=det_r,
        region_names=["ambient", "skin", "fat", "uterus", "amniotic", "fetal_head", "placenta"],
        fiber_radius=0.2, fiber_na=0.22, compat=0)


WORKLOADS = {"plain_slab": plain_slab, "curved_abdomen": curved_abdomen,
             "curved_abdomen_940": lambda n_photons=10_000_000: curved_abdomen(n_photons, 940),
             "deformed_abdomen": deformed_abdomen}


# ------------------------------------------------------------------ batched workload
# Molar extinction coefficients of oxy- and deoxyhaemoglobin [cm^-1 / M] at the two
# wavelengths, rounded from S. Prahl's public compilation of hemoglobin absorption.
# Inputs of the synthetic benchmark, not measurements.
HB_EXTINCTION = {660: (319.6, 3226.56), 940: (1214.0, 693.44)}
HB_MOLAR = 150.0 / 64500.0            # whole blood: 150 g/L haemoglobin, 64.5 kg/mol
# per-region background absorption [1/mm] and share of the drawn blood fraction
BACKGROUND_MUA = {660: [0.0, 0.005, 0.002, 0.005, 0.001, 0.005], 940: [0.0, 0.008, 0.004, 0.008, 0.001, 0.008]}
BLOOD_SHARE = [0.0, 1.0, 0.5, 1.5, 0.0, 1.0]
MATERNAL, FETAL = (1, 2, 3), (5,)


def blood_mua(spo2: float, wavelength: int) -> float:
    """Absorption coefficient of whole blood [1/mm] at saturation spo2 (0..1)."""
    e_ox, e_de = HB_EXTINCTION[int(wavelength)]
    return float(np.log(10.0) * (spo2 * e_ox + (1.0 - spo2) * e_de) * HB_MOLAR / 10.0)


def tissue_table(wavelength: int, spo2_maternal: float, spo2_fetal: float, bf_maternal: float, bf_fetal: float,
                 mus_scale=None) -> np.ndarray:
    """(n, mua, mus, g) per abdomen region: mua = background + blood share x blood
    fraction x blood absorption at the region's saturation; mus = base x mus_scale."""
    base = np.array(ABDOMEN_MEDIA[int(wavelength)], F)
    nm = base.copy()
    for r in range(1, base.shape[0]):
        mua = BACKGROUND_MUA[int(wavelength)][r]
        if r in MATERNAL:
            mua += BLOOD_SHARE[r] * bf_maternal * blood_mua(spo2_maternal, wavelength)
        elif r in FETAL:
            mua += BLOOD_SHARE[r] * bf_fetal * blood_mua(spo2_fetal, wavelength)
        else:
            mua = base[r, 1]
        nm[r, 1] = mua
        if mus_scale is not None and r != 4:
            nm[r, 2] = base[r, 2] * mus_scale[r]
    return nm


@dataclass
class BatchSpec:
    meshes: list                # Workloads (one per mesh; same source and tally layout)
    instances: list             # dicts: mesh, wavelength, nmuasg, n_photons, first, spo2_m, spo2_f


def batched_abdomen(n_instances: int = 512, budget=(1e6, 1e8), n_variants: int = 8, freq: int = 45,
                    variant_freq: int = 30, seed: int = 3) -> BatchSpec:
    """The batched forward workload: the curved-abdomen mesh plus n_variants meshes with
    fetal-head depth U(30, 70) mm and fat thickness in [5, 25] mm (reduced tessellation),
    and n_instances optical-property draws -- fetal SpO2 U(30, 70) %, maternal SpO2
    U(90, 100) %, blood fractions U(2, 8) %, mus lognormal (sigma 0.2) around each region's
    base value -- alternating 660 and 940 nm, with photon budgets log-uniform in
    `budget`.  Instance i uses mesh i mod (n_variants + 1)."""
    rng = np.random.default_rng(seed)
    meshes_ = [curved_abdomen(wavelength=660, freq=freq)]
    for _ in range(n_variants):
        depth = float(np.round(rng.uniform(30.0, 70.0), 1))
        lo = float(np.round(rng.uniform(5.0, 15.0), 1))
        hi = float(np.round(min(25.0, lo + rng.uniform(5.0, 10.0)), 1))
        # the head must clear the uterine wall (skin 2 + fat up to hi + uterus 10 mm) by 2 mm;
        # a shallower draw is redrawn (none is for the default seed)
        while depth < 2.0 + hi + 10.0 + 2.0:
            depth = float(np.round(rng.uniform(30.0, 70.0), 1))
        meshes_.append(curved_abdomen(wavelength=660, freq=variant_freq, head_depth=depth, fat=(lo, hi)))
    out, first = [], 0
    for i in range(n_instances):
        wl = 660 if i % 2 == 0 else 940
        s_f, s_m = rng.uniform(0.30, 0.70), rng.uniform(0.90, 1.00)
        bf_m, bf_f = rng.uniform(0.02, 0.08), rng.uniform(0.02, 0.08)
        mus_scale = np.exp(0.2 * rng.standard_normal(6))
        n = int(np.exp(rng.uniform(np.log(budget[0]), np.log(budget[1]))))
        out.append({"mesh": i % len(meshes_), "wavelength": wl, "spo2_m": s_m, "spo2_f": s_f,
                    "nmuasg": tissue_table(wl, s_m, s_f, bf_m, bf_f, mus_scale), "n_photons": n, "first": first})
        first += n
    return BatchSpec(meshes_, out)
