// lp_kernel.cuh -- device-side data layout and helpers of the transport kernel.
//
// Arithmetic follows src/Simulation/MCLightPropagation.cl operation by operation
// (same operand order, IEEE division and square root, no contraction: the file is
// compiled with --fmad=false), so a photon that consumes the same random numbers
// follows the same trajectory as in the reference kernel up to the last-place
// differences of logf/cosf/acosf.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace lp {

constexpr int kMaxMedia = 64;
constexpr int kMaxDet = 32;
constexpr int kStackDepth = 64;
constexpr int kGradRegions = 8;      // regions a differentiated run may have
constexpr float kNoHit = 10000.0f;   // FindTriangleInPath's initial distance (.cl:1042)
// photons of one transport launch: the kernels index them with 32 bits
constexpr int64_t kMaxLaunchPhotons = int64_t(1) << 31;

struct Medium {
    float n, mua, mus, g;
    float mut;      // mua + mus
    float alb;      // mua / (mua + mus)
    int32_t absorbs;  // mua > 0 && mus > 0  (Absorb, .cl:841-847)
    int32_t ambient;  // mua == 0 && mus == 0 (step = distance to boundary, .cl:1405-1410)
    // precomputed factors of the fast arithmetic mode
    float inv_mut, inv_mua;
    float hg_a, hg_b, hg_c, hg_d, hg_inv2g;   // 1-g^2, 1-g, 2g, 1+g^2, 1/(2g)
    float pad_;
};

struct KParams {
    // mesh (see lp_bvh.hpp)
    const float4 *node_a, *node_b, *node_c;
    const int4 *node_d;
    const float4 *tri_a, *tri_b, *tri_c;
    const float4 *tri_attr;   // by original index: unit normal, (inner | outer << 16) bits
    int32_t n_nodes, n_tri, nodes_smem, tris_smem;
    // media
    const Medium *media;
    int32_t n_media;
    // source and frame
    float p0x, p0y, p0z, v0x, v0y, v0z;
    float poix, poiy, poiz;
    float ezx, ezy, ezz;             // eZ as given (sign test of the axis override)
    float nxx, nxy, nxz, nyx, nyy, nyz, nzx, nzy, nzz;  // normalised eX, eY, eZ
    float Rsp, distMin, exitScale, w0;
    int32_t src_type;                // 0 pencil beam (reference), 1 fibre disk + cone
    float src_radius, src_cos_max;
    // run parameters
    float chance, w_th, factor;
    int32_t fetal_id;
    uint32_t compat;
    uint32_t key0, key1, stream;
    int64_t first, n, max_steps;
    // reference tally layout
    int32_t hx, hy, sft_nx, dimR, dimAlpha, rz_nr, rz_nz;
    float dg[6];
    float inv_dr, inv_dz, inv_vdx, inv_vdy, inv_vdz;   // reciprocals for the fast mode
    // tallies (fixed point, 2^32 per unit weight)
    unsigned long long *sft, *rtd, *rz, *vox, *rbins, *region, *det, *counters;
    int32_t vox_nx, vox_ny, vox_nz;
    float vox_dx, vox_dy, vox_dz;
    int32_t n_rbins;
    float rbin_dr;
    int32_t n_det;
    float det_lo[kMaxDet], det_hi[kMaxDet];
    float *exit_rec;
    int64_t exit_cap;
    // differentiation (null: off): per (ring detector d, region r), over the photons
    // scored in ring d with surface weight s, the sums of a = s * L_r and b = s * k_r,
    // where L_r is the photon's path length and k_r its number of interactions in
    // region r: grad[5 * (d * n_media + r) + {0..4}] = sum a, sum b, sum a^2, sum b^2, sum a b
    double *grad;
    // cell grid over the mesh bounds (cubic cells of size 1 / g_inv_h), one word per cell:
    //   kCellEmpty set:   no triangle touches the cell; bits 0-15 hold a lower bound of
    //                     the distance from any point of the cell to the nearest
    //                     triangle, in units of g_unit
    //   kCellEmpty clear: bits 0-23 = first entry in cell_refs, bits 24-30 = number of
    //                     triangles touching the cell (kCellDense: too many, use the BVH)
    // cell_refs holds BVH-order triangle indices.  Null cell_word: BVH queries only.
    const uint32_t *cell_word;
    const int32_t *cell_refs;   // null: the words carry safety bounds only
    int64_t n_cell_refs;
    float g_ox, g_oy, g_oz, g_inv_h, g_unit, g_eps;
    int32_t g_nx, g_ny, g_nz;
    // a cell's list holds every triangle touching the cell widened by g_margin + g_eps on
    // every side; g_h is the cell edge; step_eps bounds the rounding of one position update
    float g_margin, g_h, step_eps;
    // production arithmetic: distance a photon is moved off a face after a boundary event,
    // and the barycentric tolerance of the hit test (both 0 in the reference arithmetic)
    float boundary_push, tri_eps;
    // 1: absorption deposits are summed per cell across the warp before the atomic adds
    int32_t agg_tallies;
    // scratch: photon work counter
    unsigned long long *work;
};

// A batch: many instances (one KParams each) traced by one persistent launch.
constexpr int kBatchMedia = kGradRegions;   // regions per instance in a batch
struct BatchParams {
    const KParams *inst;             // [n_inst] per-instance parameters (device memory)
    unsigned long long *claimed;     // [n_inst] photon indices handed out so far
    int32_t *frontier;               // lowest instance that may still have unclaimed photons
    int32_t n_inst;
};

// Bounds checks of the debug build (compiled with -DLP_DEBUG into liblpcuda_debug.so):
// an index outside its array is counted in the counter slot LP_C_BOUNDS (13) and the
// access is skipped, so a bad index is reported instead of reading or writing past an
// allocation.  The release build compiles every check to `true`.
constexpr int kBoundsCounter = 13;
__device__ __forceinline__ bool in_range_dbg(unsigned long long *dbg, long long i, long long n)
{
    const bool ok = i >= 0 && i < n;
    if (!ok && dbg) atomicAdd(dbg, 1ull);
    return ok;
}
#ifdef LP_DEBUG
#define LP_IN_RANGE(dbg, i, n) ::lp::in_range_dbg((dbg), (long long)(i), (long long)(n))
#else
#define LP_IN_RANGE(dbg, i, n) true
#endif


constexpr uint32_t kCellEmpty = 0x80000000u;
constexpr uint32_t kCellDense = 127u;
constexpr int kLocalMaxCells = 8;   // larger segment boxes go to the BVH

// The cell word at p; points outside the grid read as an empty cell with bound 0.
__device__ __forceinline__ uint32_t cell_at(const KParams &P, float px, float py, float pz)
{
    if (!P.cell_word) return kCellEmpty;
    const int ix = (int)floorf((px - P.g_ox) * P.g_inv_h);
    const int iy = (int)floorf((py - P.g_oy) * P.g_inv_h);
    const int iz = (int)floorf((pz - P.g_oz) * P.g_inv_h);
    if (ix < 0 || iy < 0 || iz < 0 || ix >= P.g_nx || iy >= P.g_ny || iz >= P.g_nz) return kCellEmpty;
    return __ldg(P.cell_word + ((int64_t)iz * P.g_ny + iy) * P.g_nx + ix);
}

// Distance from p to the nearest face of the cell containing it (0 outside the grid):
// the smallest of the fractional cell coordinates and their complements, times h.
__device__ __forceinline__ float cell_face_distance(const KParams &P, float px, float py, float pz)
{
    const float fx = (px - P.g_ox) * P.g_inv_h, fy = (py - P.g_oy) * P.g_inv_h, fz = (pz - P.g_oz) * P.g_inv_h;
    const float rx = fx - floorf(fx), ry = fy - floorf(fy), rz = fz - floorf(fz);
    const float d = fminf(fminf(fminf(rx, 1.0f - rx), fminf(ry, 1.0f - ry)), fminf(rz, 1.0f - rz));
    return fmaxf(d, 0.0f) * P.g_h;
}

// Conservative distance from p to the nearest triangle (0 near a surface).
__device__ __forceinline__ float safe_distance(const KParams &P, uint32_t word)
{
    return (word & kCellEmpty) ? (float)(word & 0xffffu) * P.g_unit : 0.0f;
}

// ----------------------------------------------------------------- Philox4x32-10
__device__ __forceinline__ void philox4x32_10(uint32_t &c0, uint32_t &c1, uint32_t &c2, uint32_t &c3,
                                              uint32_t k0, uint32_t k1)
{
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t hi0 = __umulhi(0xD2511F53u, c0), lo0 = 0xD2511F53u * c0;
        const uint32_t hi1 = __umulhi(0xCD9E8D57u, c2), lo1 = 0xCD9E8D57u * c2;
        const uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
        c0 = n0;
        c1 = lo1;
        c2 = n2;
        c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}

// One Philox block per event: counter (photon lo, photon hi, event, stream), key =
// seed.  Event 0 samples the source, loop iteration i is event i + 1.  The four words
// are the event's draw slots (step, Fresnel or polar angle, azimuth, roulette), each
// mapped to ((x >> 8) | 1) * 2^-24, a uniform in (0, 1) that is never 0.
struct EventRng {
    float u0, u1, u2, u3;
    __device__ __forceinline__ void draw(uint64_t pid, uint32_t event, uint32_t stream, uint32_t k0, uint32_t k1)
    {
        uint32_t c0 = (uint32_t)pid, c1 = (uint32_t)(pid >> 32), c2 = event, c3 = stream;
        philox4x32_10(c0, c1, c2, c3, k0, k1);
        u0 = __uint2float_rn((c0 >> 8) | 1u) * 0x1.0p-24f;
        u1 = __uint2float_rn((c1 >> 8) | 1u) * 0x1.0p-24f;
        u2 = __uint2float_rn((c2 >> 8) | 1u) * 0x1.0p-24f;
        u3 = __uint2float_rn((c3 >> 8) | 1u) * 0x1.0p-24f;
    }
};

// ------------------------------------------------------------- small vectors
struct V3 { float x, y, z; };
__device__ __forceinline__ V3 v3(float x, float y, float z) { return V3{x, y, z}; }
__device__ __forceinline__ float dot3(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3 cross3(V3 a, V3 b)
{
    return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ V3 scl3(float s, V3 a) { return v3(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ V3 add3(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ V3 sub3(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
// normalize(): v / |v|, zero vector unchanged (OpenCL semantics)
__device__ __forceinline__ V3 norm3(V3 v)
{
    const float l = sqrtf(dot3(v, v));
    if (l == 0.0f) return v;
    return v3(v.x / l, v.y / l, v.z / l);
}
__device__ __forceinline__ float sign_cl(float x)
{
    if (x > 0.0f) return 1.0f;
    if (x < 0.0f) return -1.0f;
    if (x != x) return 0.0f;
    return x;
}
__device__ __forceinline__ unsigned long long fix32(float w)
{
    return (w > 0.0f) ? __float2ull_rn(w * 4294967296.0f) : 0ull;
}
__device__ __forceinline__ int trunc_sat(float q)
{
    if (q != q) return 0;
    if (q > 1e9f) return 1000000000;
    if (q < -1e9f) return -1000000000;
    return (int)q;
}
__device__ __forceinline__ int trunc_sat_d(double q)
{
    if (q != q) return 0;
    if (q > 1e9) return 1000000000;
    if (q < -1e9) return -1000000000;
    return (int)q;
}

// ------------------------------------------------------------- BVH query
// Nearest triangle along (p, v) with t in (0, bound] and t < 10000, excluding
// ref_tri; equal distances resolve to the lower original index.  Returns the
// original index or -1; *t_out = distance or 10000.
struct MeshView {
    const float4 *na, *nb, *nc;
    const int4 *nd;
    const float4 *ta, *tb, *tc;
    const float4 *s_na, *s_nb, *s_nc;
    const int4 *s_nd;
    const float4 *s_ta, *s_tb, *s_tc;
    int32_t nodes_smem, tris_smem;
    int32_t n_nodes, n_tri;          // array sizes for the debug build's bounds checks
    // barycentric tolerance of the hit test: 0 is the reference's test; a few 1e-6 (the
    // production arithmetic) lets neighbouring triangles overlap along their shared
    // edges, so no ray slips through the float gap between them
    float tri_eps;
    unsigned long long *dbg;         // its counter of skipped accesses (may be null)
};

__device__ __forceinline__ void test_tri(const MeshView &M, int j, V3 p, V3 v, int ref_tri, float &best,
                                         int &bid)
{
    if (!LP_IN_RANGE(M.dbg, j, M.n_tri)) return;
    float4 a, b, c;
    if (j < M.tris_smem) {
        a = M.s_ta[j]; b = M.s_tb[j]; c = M.s_tc[j];
    } else {
        a = __ldg(M.ta + j); b = __ldg(M.tb + j); c = __ldg(M.tc + j);
    }
    const int o = __float_as_int(c.y);
    if (o == ref_tri) return;
    const V3 Mv = v3(a.x, a.y, a.z), E = v3(a.w, b.x, b.y), F = v3(b.z, b.w, c.x);
    const V3 G = sub3(p, Mv);
    const V3 GE = cross3(G, E), VF = cross3(v, F);
    float t = dot3(GE, F);
    const float w = dot3(VF, E);
    float k = dot3(VF, G);
    float l = dot3(GE, v);
    // Division-free filter, looser than the exact test below: t, k, l must share the
    // sign of w, |k| + |l| may not exceed |w| and |t| may not exceed best * |w| (each
    // with a relative margin far above the rounding of the divided values).  Only
    // candidates that pass pay for the three IEEE divisions of the reference test.
    const float aw = fabsf(w);
    const float ek = M.tri_eps * aw;
    const bool sgn = (w > 0.0f) ? (t > 0.0f && k >= -ek && l >= -ek) : (t < 0.0f && k <= ek && l <= ek);
    if (!sgn || fabsf(k) + fabsf(l) > aw * (1.0001f + 3.0f * M.tri_eps) || fabsf(t) > best * aw * 1.0001f) return;
    t = t / w;
    k = k / w;
    l = l / w;
    if (t > 0.0f && t < kNoHit && k >= -M.tri_eps && l >= -M.tri_eps && (k + l) < 1.0f + M.tri_eps &&
        (t < best || (t == best && o < bid))) {
        best = t;
        bid = o;
    }
}

// test_tri plus a lower bound of the distance from p to the triangle: the distance to
// its plane, |(G x E) . F| / |E x F|, less a bound of the rounding of that product
// (tri_c.z = 1 / |E x F|, tri_c.w = the rounding factor per unit |G|, see lp_bvh.hpp).
// safe is lowered to that bound; the hit test is test_tri's, operation for operation.
__device__ __forceinline__ void test_tri_safe(const MeshView &M, int j, V3 p, V3 v, int ref_tri, float &best,
                                              int &bid, float &safe)
{
    if (!LP_IN_RANGE(M.dbg, j, M.n_tri)) {
        safe = 0.0f;
        return;
    }
    float4 a, b, c;
    if (j < M.tris_smem) {
        a = M.s_ta[j]; b = M.s_tb[j]; c = M.s_tc[j];
    } else {
        a = __ldg(M.ta + j); b = __ldg(M.tb + j); c = __ldg(M.tc + j);
    }
    const V3 Mv = v3(a.x, a.y, a.z), E = v3(a.w, b.x, b.y), F = v3(b.z, b.w, c.x);
    const V3 G = sub3(p, Mv);
    const V3 GE = cross3(G, E);
    float t = dot3(GE, F);
    safe = fminf(safe, fabsf(t) * c.z - c.w * (fabsf(G.x) + fabsf(G.y) + fabsf(G.z)));
    const int o = __float_as_int(c.y);
    if (o == ref_tri) return;
    const V3 VF = cross3(v, F);
    const float w = dot3(VF, E);
    float k = dot3(VF, G);
    float l = dot3(GE, v);
    const float aw = fabsf(w);
    const float ek = M.tri_eps * aw;
    const bool sgn = (w > 0.0f) ? (t > 0.0f && k >= -ek && l >= -ek) : (t < 0.0f && k <= ek && l <= ek);
    if (!sgn || fabsf(k) + fabsf(l) > aw * (1.0001f + 3.0f * M.tri_eps) || fabsf(t) > best * aw * 1.0001f) return;
    t = t / w;
    k = k / w;
    l = l / w;
    if (t > 0.0f && t < kNoHit && k >= -M.tri_eps && l >= -M.tri_eps && (k + l) < 1.0f + M.tri_eps &&
        (t < best || (t == best && o < bid))) {
        best = t;
        bid = o;
    }
}

// STACK: traversal stack entries; the host only runs a tree whose depth is below it.
template <int STACK = kStackDepth>
__device__ __noinline__ int query_nearest(const MeshView &M, V3 p, V3 v, int ref_tri, float bound,
                                             float &t_out)
{
    float best = fminf(bound, kNoHit);
    int bid = 0x7fffffff;
    const float ix = 1.0f / (fabsf(v.x) > 1e-30f ? v.x : copysignf(1e-30f, v.x));
    const float iy = 1.0f / (fabsf(v.y) > 1e-30f ? v.y : copysignf(1e-30f, v.y));
    const float iz = 1.0f / (fabsf(v.z) > 1e-30f ? v.z : copysignf(1e-30f, v.z));
    const float ox = p.x * ix, oy = p.y * iy, oz = p.z * iz;
    int stack[STACK];
    int sp = 0;
    int node = 0;
    for (;;) {
        float4 a, b, c;
        int4 d;
        if (!LP_IN_RANGE(M.dbg, node, M.n_nodes)) break;
        if (node < M.nodes_smem) {
            a = M.s_na[node]; b = M.s_nb[node]; c = M.s_nc[node]; d = M.s_nd[node];
        } else {
            a = __ldg(M.na + node); b = __ldg(M.nb + node); c = __ldg(M.nc + node); d = __ldg(M.nd + node);
        }
        // slab tests of both children against [0, best]
        float t0, t1, tn0, tf0, tn1, tf1;
        t0 = a.x * ix - ox; t1 = a.y * ix - ox;
        tn0 = fminf(t0, t1); tf0 = fmaxf(t0, t1);
        t0 = a.z * iy - oy; t1 = a.w * iy - oy;
        tn0 = fmaxf(tn0, fminf(t0, t1)); tf0 = fminf(tf0, fmaxf(t0, t1));
        t0 = c.x * iz - oz; t1 = c.y * iz - oz;
        tn0 = fmaxf(tn0, fminf(t0, t1)); tf0 = fminf(tf0, fmaxf(t0, t1));
        t0 = b.x * ix - ox; t1 = b.y * ix - ox;
        tn1 = fminf(t0, t1); tf1 = fmaxf(t0, t1);
        t0 = b.z * iy - oy; t1 = b.w * iy - oy;
        tn1 = fmaxf(tn1, fminf(t0, t1)); tf1 = fminf(tf1, fmaxf(t0, t1));
        t0 = c.z * iz - oz; t1 = c.w * iz - oz;
        tn1 = fmaxf(tn1, fminf(t0, t1)); tf1 = fminf(tf1, fmaxf(t0, t1));
        // widen the far end relative to best so rounding never culls a tie
        const float lim = best * 1.000001f + 1e-6f;
        bool h0 = fmaxf(tn0, 0.0f) <= fminf(tf0, lim);
        bool h1 = fmaxf(tn1, 0.0f) <= fminf(tf1, lim);
        if (h0 && d.x < 0) {
            const int e = ~d.x, f = e >> 3, cnt = (e & 7) + 1;
            for (int j = f; j < f + cnt; ++j) test_tri(M, j, p, v, ref_tri, best, bid);
            h0 = false;
        }
        if (h1 && d.y < 0) {
            const int e = ~d.y, f = e >> 3, cnt = (e & 7) + 1;
            for (int j = f; j < f + cnt; ++j) test_tri(M, j, p, v, ref_tri, best, bid);
            h1 = false;
        }
        if (h0 && h1) {
            const bool first0 = tn0 <= tn1;
            if (sp < STACK) stack[sp++] = first0 ? d.y : d.x;
            node = first0 ? d.x : d.y;
        } else if (h0) {
            node = d.x;
        } else if (h1) {
            node = d.y;
        } else {
            if (sp == 0) break;
            node = stack[--sp];
        }
    }
    if (bid == 0x7fffffff) {
        t_out = kNoHit;
        return -1;
    }
    t_out = best;
    return bid;
}

// The same query answered from the cell grid when the segment [p, p + bound v] is short:
// every triangle that touches a cell overlapping the segment's bounding box (widened by
// g_eps) is tested with test_tri, so the candidate set holds every triangle the test can
// accept within the bound, and the result (nearest t, then lowest original index) is
// the BVH's bit for bit.  Boxes of more than kLocalMaxCells cells, or a dense cell, go
// to query_nearest; *used_bvh reports which path answered.
template <int STACK = kStackDepth>
__device__ __forceinline__ int cell_query(const KParams &P, const MeshView &M, V3 p, V3 v, int ref_tri,
                                          float bound, float &t_out, bool &used_bvh)
{
    used_bvh = true;
    if (!P.cell_refs || !(bound < kNoHit)) return query_nearest<STACK>(M, p, v, ref_tri, bound, t_out);
    const float e = P.g_eps;
    const float qx = p.x + bound * v.x, qy = p.y + bound * v.y, qz = p.z + bound * v.z;
    const int nx = P.g_nx, ny = P.g_ny, nz = P.g_nz;
    const int x0 = min(max((int)floorf((fminf(p.x, qx) - e - P.g_ox) * P.g_inv_h), 0), nx - 1);
    const int x1 = min(max((int)floorf((fmaxf(p.x, qx) + e - P.g_ox) * P.g_inv_h), 0), nx - 1);
    const int y0 = min(max((int)floorf((fminf(p.y, qy) - e - P.g_oy) * P.g_inv_h), 0), ny - 1);
    const int y1 = min(max((int)floorf((fmaxf(p.y, qy) + e - P.g_oy) * P.g_inv_h), 0), ny - 1);
    const int z0 = min(max((int)floorf((fminf(p.z, qz) - e - P.g_oz) * P.g_inv_h), 0), nz - 1);
    const int z1 = min(max((int)floorf((fmaxf(p.z, qz) + e - P.g_oz) * P.g_inv_h), 0), nz - 1);
    if ((x1 - x0 + 1) * (y1 - y0 + 1) * (z1 - z0 + 1) > kLocalMaxCells)
        return query_nearest<STACK>(M, p, v, ref_tri, bound, t_out);
    float best = bound;
    int bid = 0x7fffffff;
    for (int z = z0; z <= z1; ++z)
        for (int y = y0; y <= y1; ++y)
            for (int x = x0; x <= x1; ++x) {
                const uint32_t w = __ldg(P.cell_word + ((int64_t)z * ny + y) * nx + x);
                if (w & kCellEmpty) continue;
                uint32_t cnt = (w >> 24) & 127u;
                if (cnt == kCellDense) return query_nearest<STACK>(M, p, v, ref_tri, bound, t_out);
                if (!LP_IN_RANGE(M.dbg, (int64_t)(w & 0xffffffu) + cnt - 1, P.n_cell_refs)) cnt = 0;
                const int32_t *r = P.cell_refs + (w & 0xffffffu);
                for (uint32_t k = 0; k < cnt; ++k) test_tri(M, __ldg(r + k), p, v, ref_tri, best, bid);
            }
    used_bvh = false;
    if (bid == 0x7fffffff) {
        t_out = kNoHit;
        return -1;
    }
    t_out = best;
    return bid;
}

// The transport's query over the cell lists, one loop for both cases (one inlined copy of
// the triangle test):
//   * the step stays within the photon's own widened cell (word: its list word, not
//     dense): that cell's list alone decides it.  The list holds every triangle touching
//     the cell widened by g_margin + g_eps, so an unlisted triangle lies at least
//     g_margin + dface from p (dface: distance from p to the cell's faces), and no
//     segment from p of length <= reach = g_margin + dface - g_eps can reach one.  `safe`
//     (coming in with a lower bound already known, the photon's carried one) is raised to
//     a lower bound of the distance from p to every triangle: reach for the unlisted ones,
//     their plane distance (test_tri_safe) for the listed ones, 0 on a triangle
//     (ref_tri >= 0);
//   * otherwise the lists of the cells the segment's box covers (at most kLocalMaxCells),
//     as cell_query; longer segments and dense cells go to the BVH.  The bound of the own
//     list would not outlast such a step (it is at most that list's reach), so `safe`
//     stays as it is.
// Same candidates, test and tie-break as cell_query and the BVH: the same hit.
template <int STACK = kStackDepth>
__device__ __forceinline__ int grid_query(const KParams &P, const MeshView &M, V3 p, V3 v, int ref_tri, float bound,
                                          uint32_t word, float &t_out, float &safe, bool &used_bvh)
{
    used_bvh = true;
    if (!P.cell_refs) return query_nearest<STACK>(M, p, v, ref_tri, bound, t_out);
    const int nx = P.g_nx, ny = P.g_ny, nz = P.g_nz;
    const bool listed = !(word & kCellEmpty) && ((word >> 24) & 127u) != kCellDense;
    const bool own = listed && bound <= P.g_margin + cell_face_distance(P, p.x, p.y, p.z) - P.g_eps;
    int x0, x1, y0, y1, z0, z1;
    if (own) {
        x0 = x1 = (int)floorf((p.x - P.g_ox) * P.g_inv_h);
        y0 = y1 = (int)floorf((p.y - P.g_oy) * P.g_inv_h);
        z0 = z1 = (int)floorf((p.z - P.g_oz) * P.g_inv_h);
    } else {
        if (!(bound < kNoHit)) return query_nearest<STACK>(M, p, v, ref_tri, bound, t_out);
        const float e = P.g_eps;
        const float qx = p.x + bound * v.x, qy = p.y + bound * v.y, qz = p.z + bound * v.z;
        x0 = min(max((int)floorf((fminf(p.x, qx) - e - P.g_ox) * P.g_inv_h), 0), nx - 1);
        x1 = min(max((int)floorf((fmaxf(p.x, qx) + e - P.g_ox) * P.g_inv_h), 0), nx - 1);
        y0 = min(max((int)floorf((fminf(p.y, qy) - e - P.g_oy) * P.g_inv_h), 0), ny - 1);
        y1 = min(max((int)floorf((fmaxf(p.y, qy) + e - P.g_oy) * P.g_inv_h), 0), ny - 1);
        z0 = min(max((int)floorf((fminf(p.z, qz) - e - P.g_oz) * P.g_inv_h), 0), nz - 1);
        z1 = min(max((int)floorf((fmaxf(p.z, qz) + e - P.g_oz) * P.g_inv_h), 0), nz - 1);
        if ((x1 - x0 + 1) * (y1 - y0 + 1) * (z1 - z0 + 1) > kLocalMaxCells)
            return query_nearest<STACK>(M, p, v, ref_tri, bound, t_out);
    }
    float best = bound, s = own ? P.g_margin + cell_face_distance(P, p.x, p.y, p.z) - P.g_eps : 0.0f;
    int bid = 0x7fffffff;
    for (int z = z0; z <= z1; ++z)
        for (int y = y0; y <= y1; ++y)
            for (int x = x0; x <= x1; ++x) {
                const uint32_t w = own ? word : __ldg(P.cell_word + ((int64_t)z * ny + y) * nx + x);
                if (w & kCellEmpty) continue;
                uint32_t cnt = (w >> 24) & 127u;
                if (cnt == kCellDense) return query_nearest<STACK>(M, p, v, ref_tri, bound, t_out);
                if (!LP_IN_RANGE(M.dbg, (int64_t)(w & 0xffffffu) + cnt - 1, P.n_cell_refs)) {
                    cnt = 0;
                    s = 0.0f;
                }
                const int32_t *r = P.cell_refs + (w & 0xffffffu);
                for (uint32_t k = 0; k < cnt; ++k) test_tri_safe(M, __ldg(r + k), p, v, ref_tri, best, bid, s);
            }
    used_bvh = false;
    if (own) safe = fmaxf(safe, ref_tri >= 0 ? 0.0f : fmaxf(s - P.g_eps, 0.0f));
    if (bid == 0x7fffffff) {
        t_out = kNoHit;
        return -1;
    }
    t_out = best;
    return bid;
}

}  // namespace lp
