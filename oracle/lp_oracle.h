/*
 * lp_oracle.h -- CPU oracle for the LightPropagation photon-transport path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker, never the product: only the
 * test-suite, the smoke check and the CPU-baseline leg of the benchmark load it.
 * The CUDA library under lightpropagation_b200/ neither links nor includes it.
 *
 * It is a plain-C, FP32 restatement of the reference kernel
 *   src/Simulation/MCLightPropagation.cl   (the per-photon transport loop)
 * and of the host-side binning of the reference launcher
 *   src/Simulation/CalculatePropagation.cpp:120-243, 1553-1684,
 * written with brute-force O(T) triangle search exactly like the reference.
 * Every function cites the reference lines it follows.
 *
 * Parity pin: the restatement is checked bit-for-bit against the reference's own
 * kernel source compiled for the CPU (oracle/build_ref.py -> oracle/_ref/) on the
 * reference's shipped models, in the reference's sequential-stream RNG mode,
 * and against golden fixtures under tests/golden/ produced by that build.
 *
 * RNG modes
 *   LPO_RNG_RAN3_SHARED  one float-state ran3 stream carried from photon to photon
 *                        (the reference kernel run one work-item at a time,
 *                        MCLightPropagation.cl:1204-1259, PSNR.cpp:116-148)
 *   LPO_RNG_RAN3_PHOTON  one float-state ran3 stream per photon, seeded from
 *                        (seed, photon index); removes the reference's
 *                        cross-work-group stream sharing, used for the CPU baseline
 *   LPO_RNG_PHILOX       Philox4x32-10 with the CUDA path's counter layout, so the
 *                        GPU and the oracle consume common random numbers
 *
 * Tallies are unsigned 64-bit fixed point with 2^32 units per unit photon weight
 * (round to nearest even), the same encoding as the CUDA path, so integer sums are
 * exact and independent of photon order and thread count.
 */
#ifndef LP_ORACLE_H
#define LP_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { LPO_RNG_RAN3_SHARED = 0, LPO_RNG_RAN3_PHOTON = 1, LPO_RNG_PHILOX = 2 };

/* Reference behaviours that are deterministic but physically questionable. */
#define LPO_COMPAT_EXIT_RSP       0x1u /* exit weight times (1-Rsp), .cl:1000-1008          */
#define LPO_COMPAT_AXIS_NORMAL    0x2u /* normal := +-eZ within 0.01 of the axis, .cl:1493  */
#define LPO_COMPAT_SIGNED_FRESNEL 0x4u /* Fresnel with signed cos(incidence), .cl:889-896   */
#define LPO_COMPAT_ALL            0x7u
#define LPO_MAX_MEDIA             64   /* regions the perturbation-MC sums can track */

/* counters[] slots */
enum {
    LPO_C_SCATTER = 0,  /* scatter/absorb events (E_s)                            */
    LPO_C_BOUNDARY,     /* boundary interactions (E_b)                            */
    LPO_C_QUERY,        /* nearest-triangle queries (E_q) = loop iterations       */
    LPO_C_ROULETTE,     /* roulette draws                                         */
    LPO_C_MISS,         /* boundary step with no triangle hit (photon dropped)    */
    LPO_C_CAPPED,       /* photons stopped by the step cap                        */
    LPO_C_RZ_DROP,      /* absorption deposits outside the r-z grid               */
    LPO_C_VOX_DROP,     /* absorption deposits outside the voxel grid             */
    LPO_C_PHOTONS,      /* photons traced                                         */
    LPO_C_DRAWS,        /* uniform numbers consumed                               */
    LPO_C_MISMATCH,     /* boundary events on a face that does not border the photon's region */
    LPO_NCOUNTERS = 16
};

typedef struct lpo_problem {
    /* mesh in the reference launcher's AoS layouts (CalculatePropagation.cpp:541-667) */
    int32_t n_tri;
    const float *tri;       /* 9 floats per triangle: K, L, M vertices          */
    const float *nrm;       /* 3 floats per triangle (normalised in the kernel)  */
    const int32_t *med;     /* 2 ints per triangle: inner, outer region          */
    int32_t n_media;
    const float *nmuasg;    /* 4 floats per region: n, mua, mus, g (.cpp:427-451) */
    /* source (Emitter.cpp:186-339) */
    float p_start[3];
    float v_start[3];
    float ep0xyz[12];       /* POI, eX, eY, eZ                                    */
    /* reference tally layout inputs */
    float dimensions[3];    /* model extent, config <dimensions>                 */
    float det_grid[6];      /* x, y, z, r, phi, rho (config <DetectionGrid>)     */
    int32_t fetal_id;
    float chance, w_threshold, factor;
    /* run control */
    uint32_t compat;
    int32_t rng_mode;
    uint64_t seed;
    uint32_t stream;        /* Philox counter word 3 (instance id in batches)    */
    int64_t max_steps;      /* per-photon loop cap; <= 0 means no cap            */
    /* tallies added by the build */
    int32_t vox_n[3];
    float vox_d[3];
    int32_t n_rbins;
    float rbin_dr;
    int32_t n_det;
    const float *det_r;     /* n_det x (r_lo, r_hi) annuli of the exit radius    */
    /* source extension (no reference counterpart): 0 = pencil beam as in the
     * reference, 1 = fibre: start point uniform on a disk of radius src_radius
     * around p_start in the (eX, eY) plane, direction uniform in solid angle
     * within the cone cos(theta) >= src_cos_max around eZ.  Four draws
     * (r, phi, cos theta, psi) open the photon's stream. */
    int32_t src_type;
    float src_radius, src_cos_max;
} lpo_problem;

typedef struct lpo_geometry {
    int32_t dimx, dimy, dimz, dimR, dimAlpha;
    int32_t sft_nx, sft_ny;   /* (2*(dimx/2)+1), (2*(dimy/2)+1) */
    int32_t rz_nr, rz_nz;     /* 2*dimR+1, dimz+1               */
    int32_t kernel_dimR;      /* dimR as the kernel computes it (.cl:263) */
} lpo_geometry;

typedef struct lpo_tallies {
    uint64_t *sft;      /* [sft_ny][sft_nx][3]  surf, fetal, trans   (CP.cpp:1553-1584) */
    uint64_t *rtd;      /* [dimAlpha][dimR][3]                        (CP.cpp:1587-1626) */
    uint64_t *rz;       /* [rz_nz][rz_nr][2]    absorbed, absorbed/mua                  */
    uint64_t *vox;      /* [nz][ny][nx]         absorbed                                */
    uint64_t *rbins;    /* [n_rbins][2]         surface, transmitted exit weight        */
    uint64_t *region;   /* [n_media]            absorbed per region                     */
    uint64_t *det;      /* [n_det][2]           sum w, sum w^2 of surface exits         */
    uint64_t counters[LPO_NCOUNTERS];
    float *exit_rec;    /* optional [n][8] per-photon record (.cl:119-130)              */
    float *rz_ref;      /* optional reference-layout r-z buffer, see lpo_rz_ref_layout  */
    int64_t rz_ref_cells;   /* cells (3 floats each) in rz_ref                          */
    int64_t rz_ref_offset;  /* cell index of the reference's cell 0 inside rz_ref       */
    /* optional perturbation-MC sums [n_det][n_media][5] (FP64): over the photons
     * scored in ring d with surface weight s, with L_r / k_r the photon's path length /
     * interaction count in region r: sum s L_r, sum s k_r, sum (s L_r)^2,
     * sum (s k_r)^2, sum (s L_r)(s k_r).  The derivative of the ring signal
     * (mean s per launched photon) is -sum s L_r / (factor N) for mua_r and
     * (sum s k_r / mus_r - sum s L_r / factor) / N for mus_r. */
    double *grad;
} lpo_tallies;

/* Philox4x32-10 block function (Salmon et al., SC'11). */
void lpo_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

/* PSNR::InitRand3 + GetRan3Array + GetInextInextp (PSNR.cpp:116-148, 173-237):
 * state56 receives the 56-entry table as floats, inext3 = {inext, inextp, 0}. */
void lpo_ran3_init(int32_t seed, float state56[56], int32_t inext3[3]);

/* One draw of the kernel's float-state ran3 (MCLightPropagation.cl:1204-1237). */
float lpo_ran3_draw(float state56[56], int32_t inext3[3]);

/* Image extents of CalculatePropagation::InitLogVectors (CP.cpp:120-243). */
void lpo_geometry_of(const float dimensions[3], const float det_grid[6], lpo_geometry *g);

/* Specular reflectance (MCLightPropagation.cl:273-299). */
float lpo_rspecular(const float *nmuasg);

/* Unpolarised Fresnel reflectance (MCLightPropagation.cl:857-907). */
float lpo_fresnel(float n1, float n2, float cos_in);

/* Henyey-Greenstein cos(theta) as in VScatter (MCLightPropagation.cl:625-634). */
float lpo_hg_cos_theta(float g, float xi);

/* Nearest triangle along (p, v) excluding ref_tri, brute force
 * (MCLightPropagation.cl:1037-1093).  Returns the index or -1, *t_out = distance. */
int32_t lpo_find_triangle(const float *tri, int32_t n_tri, int32_t ref_tri,
                          const float p[3], const float v[3], float *t_out);

/* Trace photons [first, first+n).  nthreads <= 0 uses all cores.  For
 * LPO_RNG_RAN3_SHARED the run is sequential and ran3_state/ran3_inext carry the
 * stream in and out (as the reference's rand3Arr/inxtInxtpLocked buffers do).
 * Tally arrays must be zeroed by the caller; results are added.  Returns 0. */
int lpo_run(const lpo_problem *P, int64_t first, int64_t n, int nthreads,
            float *ran3_state, int32_t *ran3_inext, lpo_tallies *T);

/* Fixed-point encoding of a non-negative weight. */
uint64_t lpo_fix(float w);

/* ---- FP64 error oracle (lp_oracle64.c) ------------------------------------------
 * The same physics, tallies and Philox draw layout as lpo_run with every quantity in
 * double precision; the nearest-triangle search runs over a bounding-volume tree and
 * returns the brute-force scan's answer (nearest t, then lowest index).  Only the
 * LPO_RNG_PHILOX mode exists.  exit_rec receives the records rounded to float; rz_ref
 * is not produced.  Tally arrays must be zeroed by the caller; results are added. */
typedef struct lpo64_mesh lpo64_mesh;
lpo64_mesh *lpo64_mesh_build(const float *tri, int32_t n_tri);
void lpo64_mesh_free(lpo64_mesh *m);
/* Nearest triangle along (p, v) with 0 < t <= bound and t < 10000, ref_tri excluded:
 * through the tree, and by the brute-force scan of .cl:1037-1093 in double. */
int32_t lpo64_mesh_query(const lpo64_mesh *m, int32_t ref_tri, const double p[3], const double v[3],
                         double bound, double *t_out);
int32_t lpo64_find_triangle(const float *tri, int32_t n_tri, int32_t ref_tri, const double p[3],
                            const double v[3], double bound, double *t_out);
double lpo64_fresnel(double n1, double n2, double cos_in);
/* Trace photons [first, first+n) in FP64; mesh may be NULL (built and freed here).
 * Returns 0, or 1 if the problem is not in the Philox mode or has too many regions. */
int lpo64_run(const lpo_problem *P, const lpo64_mesh *mesh, int64_t first, int64_t n, int nthreads,
              lpo_tallies *T);

#ifdef __cplusplus
}
#endif
#endif
