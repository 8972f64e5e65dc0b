/*
 * lpcuda.h -- C ABI of the B200 photon-transport library (liblpcuda.so).
 *
 * Drop-in boundary for the hot path of LightPropagation: the OpenCL kernel
 * MCLightPropagation (src/Simulation/MCLightPropagation.cl:1262-1269) and the
 * launcher class that feeds it (src/Simulation/CalculatePropagation.hpp:212-388).
 * Each entry point below names the reference interface it replaces.
 *
 * Conventions
 *   - Plain pointers and sizes only; every call returns an int status
 *     (LP_OK == 0, the reference's SUCCESS, CalculatePropagation.cpp:23-25).
 *     Nothing is thrown across the ABI.  lp_last_error() gives the message.
 *   - Inputs are deep-copied at set time (like the reference setters,
 *     CalculatePropagation.cpp:351-667); the caller keeps ownership of its arrays.
 *   - Output arrays returned by lp_get_tallies() are owned by the context and stay
 *     valid until the next lp_run, lp_run_async, lp_zero_tallies or lp_destroy
 *     on that context.
 *   - One context per host thread; calls on one context must be serialised.
 *     Each context owns one CUDA stream.
 *   - Tallies are unsigned 64-bit fixed point, LP_FIX_ONE units per unit photon
 *     weight, so sums are exact and identical from run to run and for any grid or
 *     block shape.
 */
#ifndef LPCUDA_H
#define LPCUDA_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LP_OK            0
#define LP_ERR_INVALID   1  /* bad argument                                  */
#define LP_ERR_CUDA      2  /* CUDA runtime error                            */
#define LP_ERR_STATE     3  /* call out of order (e.g. run before set_mesh)  */
#define LP_ERR_NOMEM     4  /* allocation failed                             */
#define LP_ERR_RANGE     5  /* size beyond a supported maximum               */
#define LP_ERR_TIMEOUT   6  /* a device-side wait gave up                    */

#define LP_FIX_ONE 4294967296.0 /* 2^32 */

/* Reference behaviours kept by default (deterministic quirks of the reference). */
#define LP_COMPAT_EXIT_RSP       0x1u /* exit weight times (1-Rsp), MCLightPropagation.cl:1000-1008  */
#define LP_COMPAT_AXIS_NORMAL    0x2u /* normal := +-eZ within 0.01 of the axis, .cl:1493-1498      */
#define LP_COMPAT_SIGNED_FRESNEL 0x4u /* Fresnel with the signed incidence cosine, .cl:889-896      */
#define LP_COMPAT_ALL            0x7u

/* Counter slots of lp_tallies.counters */
enum {
    LP_C_SCATTER = 0, LP_C_BOUNDARY, LP_C_QUERY, LP_C_ROULETTE, LP_C_MISS, LP_C_CAPPED,
    LP_C_RZ_DROP, LP_C_VOX_DROP, LP_C_PHOTONS, LP_C_DRAWS, LP_C_SAFE_SKIP, LP_C_BVH_QUERY,
    LP_C_BAD_INPUT,   /* lp_run_noalloc: triangles whose region ids failed the device-side check */
    LP_C_BOUNDS,      /* bounds-checked build (liblpcuda_debug.so): accesses skipped as out of range */
    LP_C_REGION_MISMATCH, /* boundary events whose face does not border the photon's region */
    LP_C_AGG_LEADERS, /* aggregated tallies (lp_set_tally_aggregation): r-z deposit groups, one
                         atomic each; 1 - groups / deposits is the warp match rate */
    LP_NCOUNTERS = 16
};

typedef struct lp_ctx lp_ctx;

/* Tally-image extents derived like CalculatePropagation::InitLogVectors
 * (CalculatePropagation.cpp:120-243). */
typedef struct lp_geometry {
    int32_t dimx, dimy, dimz, dimR, dimAlpha;
    int32_t sft_nx, sft_ny;   /* SFT image  [-dimx/2, dimx/2] x [-dimy/2, dimy/2] */
    int32_t rz_nr, rz_nz;     /* r-z image  [-dimR, dimR] x [-dimz, 0]            */
    int32_t kernel_dimR;
} lp_geometry;

/* Host copies of the tallies of the last run(s), fixed point (LP_FIX_ONE).  */
typedef struct lp_tallies {
    const uint64_t *sft;    /* [sft_ny][sft_nx][3] surf, fetal, trans (GetSFTImage)      */
    const uint64_t *rtd;    /* [dimAlpha][dimR][3] (GetRTdImage)                          */
    const uint64_t *rz;     /* [rz_nz][rz_nr][2] absorbed, absorbed/mua (GetArz/PhirzImage) */
    const uint64_t *vox;    /* [nz][ny][nx] absorbed weight per voxel                     */
    const uint64_t *rbins;  /* [n_rbins][2] surface, transmitted exit weight by radius    */
    const uint64_t *region; /* [n_media] absorbed weight per region                       */
    const uint64_t *det;    /* [n_det][2] sum w, sum w^2 of surface exits per ring        */
    uint64_t counters[LP_NCOUNTERS];
    int64_t n_vox, n_rbins, n_region, n_det;
} lp_tallies;

/* --- context -------------------------------------------------------------- */
/* Replaces CalculatePropagation::CalculatePropagation + createContext
 * (CalculatePropagation.cpp:27-79, 1302-1335). */
int lp_create(lp_ctx **out, int device);
/* Replaces CalculatePropagation::cleanup + ~CalculatePropagation (CP.cpp:1944-2001, 82-115). */
void lp_destroy(lp_ctx *ctx);
/* Last error message of ctx (or of the calling thread when ctx is NULL). */
const char *lp_last_error(const lp_ctx *ctx);

/* --- inputs --------------------------------------------------------------- */
/* SetTriangles + SetNormals + SetInnerAndOuterTissueIndices
 * (CalculatePropagation.cpp:541-667): tri = 9 floats (K, L, M) per triangle,
 * nrm = 3 floats per triangle (normalised on use), med = (inner, outer) region ids.
 * Builds the SoA BVH.  n_tri up to 2^27. */
int lp_set_mesh(lp_ctx *ctx, int64_t n_tri, const float *tri, const float *nrm,
                const int32_t *med);
/* SetTissueProperties (CalculatePropagation.cpp:427-451): n, mua, mus, g per region
 * (the packed float4 layout of the kernel's nMuasG argument).  Up to 64 regions. */
int lp_set_media(lp_ctx *ctx, int32_t n_media, const float *nmuasg);
/* SetStartTrajectories + SetStartPoint + SetPOI + SetBasisVectors
 * (CalculatePropagation.cpp:332-339, 365-380, 760-790): p_start[3], k start
 * directions (only the first is used, as in the kernel, .cl:429-467) and the
 * 12 floats POI, eX, eY, eZ (the kernel's e_P0XYZ). */
int lp_set_source(lp_ctx *ctx, const float *p_start, const float *v_start,
                  const int32_t *v_occ, int32_t k, const float *ep0xyz);
/* Fibre source (no reference counterpart; the reference launches a pencil beam):
 * start points uniform on a disk of `radius` around p_start in the (eX, eY) plane,
 * directions uniform in solid angle within the cone of half-angle asin(na / n0)
 * about eZ (n0 = refractive index of region 0).  radius = na = 0 restores the
 * pencil beam. */
int lp_set_fiber_source(lp_ctx *ctx, float radius, float na);
/* SetDimensions + SetDetectionGridDimensions + SetFetalTissueID
 * (CalculatePropagation.cpp:536-539, 716-735, 792-794): model extent, detection
 * grid (x, y, z, r, phi, rho) and the fetal region id.  Fixes the image extents. */
int lp_set_tally_grid(lp_ctx *ctx, const float *dimensions, const float *det_grid,
                      int32_t fetal_id);
/* SetChanceForRoulette + SetWeightThreshold + SetPixelPerUnitFactor
 * (CalculatePropagation.cpp:380-397) plus the RNG seed that replaces the
 * time-seeded ran3 table (PSNR.cpp:98) and the compat switches. */
int lp_set_params(lp_ctx *ctx, float chance, float w_threshold, float factor,
                  uint64_t seed, uint32_t compat);
/* Tallies added by this library (no reference counterpart): voxel absorption grid
 * in the emitter frame, radial exit bins, ring detectors (n_det annuli r_lo, r_hi). */
int lp_set_extra_tallies(lp_ctx *ctx, const int32_t *vox_n, const float *vox_d,
                         int32_t n_rbins, float rbin_dr, int32_t n_det, const float *det_r);
/* Arithmetic of the transport kernel.  exact = 1 follows the reference kernel's
 * floating-point operations one by one (same operand order, IEEE division, no FMA
 * contraction), so with the same random numbers a photon retraces the CPU oracle's
 * trajectory; exact = 0 (default) samples the same distributions with fewer
 * operations (precomputed Henyey-Greenstein factors, direction-cosine scattering
 * update, vector refraction, reciprocal multiplies, FMA). */
int lp_set_arithmetic(lp_ctx *ctx, int exact);
/* Cell grid (no reference counterpart): a grid of at most max_cells cells over the
 * mesh bounds, built on the device once per mesh (default 2^24 cells).  A cell that
 * no triangle touches holds a lower bound of the distance to the nearest triangle: a
 * step shorter than the bound at the photon's position cannot reach a triangle, so
 * its nearest-triangle query is skipped.  A cell that triangles touch lists them: a
 * short step's query tests only the triangles of the cells around the step instead of
 * descending the BVH.  Neither changes any result.  0 disables the grid. */
int lp_set_safety_grid(lp_ctx *ctx, int64_t max_cells);
/* ---- Differentiation (no reference counterpart) ---------------------------------
 * Derivatives of the ring-detector signals S_d (mean surface weight per launched
 * photon scored in ring d of lp_set_extra_tallies) with respect to the absorption and
 * scattering coefficients of every region, accumulated in the same pass as the
 * forward run.  Each photon keeps its path length L_r and interaction count k_r per
 * region (FP32); a photon scored with weight s in ring d adds s * (-L_r / factor) to
 * dS_d/dmua_r and s * (k_r / mus_r - L_r / factor) to dS_d/dmus_r (perturbation Monte
 * Carlo).  The sums are FP64.  At most 8 regions. */
int lp_set_gradient(lp_ctx *ctx, int enable);

typedef struct lp_gradient {
    int32_t n_det, n_media;
    int64_t n_photons;        /* photons the sums cover (since the tallies were zeroed) */
    const double *signal;     /* [n_det]           S_d                                   */
    const double *signal_se;  /* [n_det]           standard error of S_d                  */
    const double *d_mua;      /* [n_det][n_media]  dS_d / dmua_r                         */
    const double *d_mus;      /* [n_det][n_media]  dS_d / dmus_r                         */
    const double *d_mua_se;   /* [n_det][n_media]  standard errors of the derivatives     */
    const double *d_mus_se;
} lp_gradient;
/* Reads the sums back and forms signals and derivatives.  The arrays are owned by
 * ctx and stay valid until the next lp_get_gradient / lp_forward / lp_destroy. */
int lp_get_gradient(lp_ctx *ctx, lp_gradient *out);
/* Forward half of an autograd-style function: zero the tallies, trace photons
 * [first, first + n) with differentiation on, and write S_d to signal[n_det]
 * (may be NULL). */
int lp_forward(lp_ctx *ctx, int64_t first, int64_t n, double *signal);
/* Backward half, the vector-Jacobian product of the last lp_forward:
 * grad_mua[r] = sum_d grad_signal[d] dS_d/dmua_r and grad_mus likewise, n_media
 * entries each. */
int lp_backward(lp_ctx *ctx, const double *grad_signal, double *grad_mua, double *grad_mus);

/* ---- Batches (no reference counterpart) -----------------------------------------
 * Many transport instances in one persistent launch, replayed as a CUDA graph.  An
 * instance is one of the batch's contexts (its mesh, source, tally layout and run
 * parameters as set on that lp_ctx) with its own optical properties, photon range and
 * tallies.  The reference traces one problem per program run
 * (CalculatePropagation.cpp:1389-1759); here wavelengths x optical-property draws x
 * meshes with uneven budgets share the GPU and drain once.  Each instance's tallies
 * equal, bit for bit, those of lp_run on its context with its media and photon range.
 * All contexts must live on the same device and share one tally layout. */
#define LP_BATCH_MAX_MEDIA 8
typedef struct lp_instance {
    int32_t context;                          /* index into the batch's contexts         */
    int32_t n_media;                          /* regions, at most LP_BATCH_MAX_MEDIA      */
    float nmuasg[4 * LP_BATCH_MAX_MEDIA];     /* n, mua, mus, g per region                */
    int64_t first;                            /* first photon id                          */
    int64_t n_photons;
} lp_instance;
typedef struct lp_batch lp_batch;
/* ctxs: n_ctx configured contexts (not owned; they must outlive the batch). */
int lp_batch_create(lp_batch **out, int32_t n_ctx, lp_ctx *const *ctxs);
void lp_batch_destroy(lp_batch *b);
const char *lp_batch_last_error(const lp_batch *b);
int lp_batch_set_instances(lp_batch *b, int32_t n_inst, const lp_instance *inst);
/* Differentiation for every instance (see lp_set_gradient). */
int lp_batch_set_gradient(lp_batch *b, int enable);
/* Instances of at least `photons` photons run as a persistent transport launch of their
 * own inside the batch's graph (the rest share the batch launch); photons <= 0: all
 * share it.  Default 2^20: the batch kernel's instance switching costs every photon a
 * little, a launch of its own costs one drain, and the two meet near 7e5 photons on the
 * abdomen.  Tallies are the same either way. */
int lp_batch_set_plain_threshold(lp_batch *b, int64_t photons);
/* Instances the current setting runs as launches of their own. */
int lp_batch_plain_count(const lp_batch *b, int32_t *count);
/* Launch configuration: -1 (default) autotunes on the first run; 0..count-1 fixes one. */
int lp_batch_config_count(void);
int lp_batch_config_info(int32_t config, int32_t *block, int32_t *min_blocks, int32_t *stack);
int lp_batch_set_config(lp_batch *b, int32_t config);
/* Autotuner: time every eligible configuration on the current instances with the
 * budgets scaled to about `photons` in total, keep the fastest.  ns_per_photon (may
 * be NULL) receives lp_batch_config_count() values, device nanoseconds per photon
 * (< 0: configuration not eligible for these meshes). */
int lp_batch_autotune(lp_batch *b, int64_t photons, int32_t *best, double *ns_per_photon);
/* Zero all instance tallies and trace every instance (one graph launch). */
int lp_batch_run(lp_batch *b);
int lp_batch_last_ms(const lp_batch *b, float *ms);
/* Ring signals S_d per instance and their relative standard errors, [n_inst][n_det]. */
int lp_batch_ring_signals(lp_batch *b, double *signal, double *rel_err);
int lp_batch_get_tallies(lp_batch *b, int32_t inst, lp_tallies *out);
int lp_batch_get_gradient(lp_batch *b, int32_t inst, lp_gradient *out);

/* Shared memory per block (bytes) for BVH nodes and triangles staged by the transport
 * kernel; what a block does not take stays L1 cache for the cell grid, tallies and the
 * rest of the mesh.  Default 8192.  No reference counterpart; results do not depend on it. */
int lp_set_smem_budget(lp_ctx *ctx, int32_t bytes);
/* Whether cells touched by triangles list them (1, default) or hold no information
 * (0: every query that the safety bound does not skip descends the BVH).  Results are
 * identical either way; lp_query_triangles follows the same setting. */
int lp_set_cell_lists(lp_ctx *ctx, int enable);
/* Margin of the cell lists, in cells (default 0.5; 0 to 4): each cell lists the
 * triangles that touch the cell widened by this margin on every side.  A wider margin
 * lets more short-step queries be answered from one cell's list and gives larger
 * distance bounds from the planes of the listed triangles, at the cost of longer lists.
 * Results do not depend on it.  No reference counterpart. */
int lp_set_cell_margin(lp_ctx *ctx, float cells);
/* Warp-aggregated absorption tallies (no reference counterpart; the reference's r-z
 * tally is a racy read-modify-write, MCLightPropagation.cl:254-271): enable = 1 makes
 * the lanes of a warp that deposit into the same r-z cell or voxel in the same step sum
 * their fixed-point values (__match_any_sync + redux.sync) so that one lane issues the
 * atomic add.  Integer sums: the tallies are identical either way. */
int lp_set_tally_aggregation(lp_ctx *ctx, int enable);
/* Per-photon step cap (watchdog); photons that reach it are stopped and counted. */
int lp_set_max_steps(lp_ctx *ctx, int64_t max_steps);
/* Keep the per-photon float8 exit records of the next runs (RecordFSTxy,
 * MCLightPropagation.cl:119-130): up to `capacity` photons, indexed by photon id
 * minus the run's first id. */
int lp_set_exit_records(lp_ctx *ctx, int64_t capacity);

/* --- run -------------------------------------------------------------------- */
/* CalculatePropagation::Init + Propagation -> ExecKernel (CP.cpp:2003-2025, 1389-1759):
 * traces photons [first, first + n) in one persistent launch (several in order when n
 * exceeds 2^31, with the same tallies) and adds their tallies.  Blocks until done. */
int lp_run(lp_ctx *ctx, int64_t first, int64_t n);
/* As lp_run but returns after the launch is queued on the context's stream. */
int lp_run_async(lp_ctx *ctx, int64_t first, int64_t n);
int lp_sync(lp_ctx *ctx);
/* Clear the accumulated tallies and counters. */
int lp_zero_tallies(lp_ctx *ctx);
/* Image extents (InitLogVectors, CP.cpp:120-243). */
int lp_get_geometry(lp_ctx *ctx, lp_geometry *out);
/* Copy the tallies to host memory owned by ctx (GetSFTImage / GetRTdImage /
 * GetArzImage / GetPhirzImage, CalculatePropagation.cpp:897-1056). */
int lp_get_tallies(lp_ctx *ctx, lp_tallies *out);
/* Checkpoint and resume (the reference carries only its ran3 table from launch to
 * launch, CalculatePropagation.cpp:1213-1215; with Philox a photon's random numbers
 * depend on the seed and its id alone, so a checkpoint is the seed, the next photon id
 * and the integer tallies).  lp_set_tallies replaces the context's tallies and counters
 * with host values in the lp_tallies layout that lp_get_tallies returns for the same
 * tally grid (sizes n_vox, n_rbins, n_region, n_det must match).  Photons [0, k) traced,
 * saved, and resumed in another context by lp_set_tallies + lp_run(ctx, k, n - k) give
 * the tallies of one run of [0, n) bit for bit. */
int lp_set_tallies(lp_ctx *ctx, const lp_tallies *in);
/* The FP64 differentiation sums of the same checkpoint, n = n_det * n_media * 5 values in
 * the layout of lp_set_gradient's sums (ring, region, 5 moments). */
int lp_get_gradient_sums(lp_ctx *ctx, double *out, int64_t n);
int lp_set_gradient_sums(lp_ctx *ctx, const double *in, int64_t n);
/* Copy n exit records (8 floats each) to out. */
int lp_get_exit_records(lp_ctx *ctx, float *out, int64_t n);
/* Device time of the last lp_run* in milliseconds (PrintTimeSpent, CP.cpp:2063-2070). */
int lp_last_kernel_ms(lp_ctx *ctx, float *ms);

/* Launch and transfer statistics of a context (PrintSimulationParams,
 * CalculatePropagation.cpp:2043-2048, extended). */
typedef struct lp_stats {
    int64_t n_tri, n_nodes;
    int32_t bvh_depth, nodes_smem, tris_smem, smem_bytes, blocks_per_sm, grid, block, num_sms;
    int64_t h2d_bytes;      /* bytes uploaded by the last lp_run* (0 if nothing changed) */
    int64_t d2h_bytes;      /* bytes copied by the last lp_get_tallies                   */
    float last_kernel_ms;
} lp_stats;
int lp_get_stats(lp_ctx *ctx, lp_stats *out);

/* Device addresses of the tally arrays (same layouts as lp_tallies), for a caller
 * that reduces them across GPUs without a host round trip.  Valid until the next
 * lp_set_tally_grid / lp_set_extra_tallies / lp_destroy. */
typedef struct lp_device_tallies {
    uint64_t *sft, *rtd, *rz, *vox, *rbins, *region, *det, *counters;
    int64_t n_sft, n_rtd, n_rz, n_vox, n_rbins, n_region, n_det, n_counters;
    void *stream;            /* the context's cudaStream_t */
    double *grad;            /* FP64 differentiation sums (lp_get_gradient_sums layout)  */
    int64_t n_grad;          /* their count; 0 while differentiation is off             */
} lp_device_tallies;
int lp_get_device_tallies(lp_ctx *ctx, lp_device_tallies *out);

/* FP32 FMA throughput of the device in TFLOP/s (2 flops per FMA), measured by a
 * dependent-FMA kernel: the roofline denominator of the transport kernel. */
int lp_fp32_peak(int device, double *tflops);

/* Throughput of 64-bit atomic adds to random slots of an L2-resident 16 MB buffer, in
 * atomics per second: the denominator of the transport kernel's L2-atomic fraction. */
int lp_l2_atomic_peak(int device, double *per_s);

/* Test hook (no reference counterpart): the device or page-locked host allocation made
 * by this library after `after` more successful ones fails as if memory were exhausted
 * (the call that needed it returns LP_ERR_NOMEM and leaves its context usable); -1
 * switches the injection off.  Process-wide. */
int lp_debug_fail_allocation(int64_t after);

/* --- transport without device allocation ------------------------------------- */
/* No counterpart in the reference.  For callers that must not allocate device memory
 * through this library: a host application whose device memory comes from its own
 * pool or arena with a fixed budget, or code that cannot afford the device-wide
 * synchronisation that cudaFree implies.  lp_run_noalloc traces photons [first, first + n_photons) with
 * the reference-arithmetic transport kernel and never calls cudaMalloc or cudaFree.
 * Its scratch (photon counter, event counters, media table and a small BVH built on
 * the device from the mesh arrays) lives in one static device array of
 * LP_NOALLOC_SCRATCH_BYTES that every GPU loading the library holds until exit.
 *   - mesh arrays are DEVICE pointers in the reference layouts (tri 9 floats, nrm 3
 *     floats, med 2 ints per triangle); region ids must lie in [0, n_media).  They are
 *     checked on the device: if any is outside, no photon is traced and
 *     counters[LP_C_BAD_INPUT] holds the number of such triangles (so pass counters to
 *     see it); lp_set_mesh rejects the same mesh with LP_ERR_INVALID;
 *   - dimensions must be finite and positive, and every image extent (dimensions /
 *     det_grid, 90 / det_grid[5]) below 2^20 cells, else LP_ERR_INVALID / LP_ERR_RANGE;
 *   - photons stop after LP_NOALLOC_MAX_STEPS steps (counted in LP_C_CAPPED);
 *   - n_photons is at most 2^31 per call (LP_ERR_RANGE beyond; an lp_instance likewise);
 *   - nmuasg is a HOST pointer (n, mua, mus, g per region), copied into kernel params;
 *   - sft, rtd, rz, region are DEVICE outputs in the lp_tallies layouts (sizes as
 *     lp_get_geometry reports for the same dimensions and grid); results are ADDED to
 *     them, so zero them first; counters (16 uint64) is optional;
 *   - sizes beyond LP_NOALLOC_MAX_TRI triangles or LP_NOALLOC_MAX_MEDIA regions are
 *     rejected with LP_ERR_RANGE.
 * The call is asynchronous on `stream` (a cudaStream_t, NULL for the default stream).
 * Each call outside stream capture looks up the scratch address on the current device
 * (after cudaDeviceReset the array may move); a call inside a capture uses the address
 * an earlier call on that device found, so make the first call on a device before any
 * stream capture.  All calls share the one scratch array, so calls that overlap on the
 * GPU race: serialise them on one stream. */
#define LP_NOALLOC_MAX_TRI 4096
#define LP_NOALLOC_MAX_MEDIA 64
#define LP_NOALLOC_MAX_STEPS 100000000   /* per-photon step cap (lp_run's default) */
#define LP_NOALLOC_SCRATCH_BYTES (384 * 1024)
typedef struct lp_noalloc_args {
    const float *tri, *nrm;
    const int32_t *med;
    int64_t n_tri;
    const float *nmuasg;
    int32_t n_media;
    float p_start[3], v_start[3], ep0xyz[12];
    float fiber_radius, fiber_cos_max;   /* fibre source; 0 and 1 for the pencil beam */
    float dimensions[3], det_grid[6];
    int32_t fetal_id;
    float chance, w_threshold, factor;
    uint64_t seed;
    uint32_t compat;
    int64_t first, n_photons;
    uint64_t *sft, *rtd, *rz, *region, *counters;
} lp_noalloc_args;
int lp_run_noalloc(const lp_noalloc_args *args, void *stream);

/* --- verification entry points ---------------------------------------------- */
/* Nearest-triangle queries through the device BVH for n rays (FindTriangleInPath,
 * MCLightPropagation.cl:1037-1093): origins/dirs 3 floats per ray, ref_tri the
 * excluded triangle per ray (or -1), t_max the query bound per ray.  Writes the
 * triangle id (-1 for none) and the distance (10000 for none). */
int lp_query_triangles(lp_ctx *ctx, int64_t n, const float *orig, const float *dir,
                       const int32_t *ref_tri, const float *t_max, int32_t *id_out,
                       float *t_out);
/* Philox4x32-10 blocks on the device: out[4*i..] = philox(ctr + (0,0,i,0), key). */
int lp_philox_blocks(int device, const uint32_t *ctr, const uint32_t *key, int64_t n,
                     uint32_t *out);

#ifdef __cplusplus
}
#endif
#endif
