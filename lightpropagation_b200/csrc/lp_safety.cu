// lp_safety.cu -- safety-distance grid over the mesh, built once per mesh on the GPU.
//
// Cell value = a lower bound, in units of `unit`, of the distance from ANY point of the
// cell to the nearest triangle: (distance from the cell centre, exact within a few cells
// of a triangle and a lower bound farther out) - (half cell diagonal) - eps, rounded
// down.  eps covers the rounding of the reference's
// ray/triangle test, which can accept intersection points a few ulp outside a
// triangle.  A transport step shorter than this bound cannot reach any triangle, so
// the bounded nearest-hit query would return "no hit": the kernel skips it and the
// result is unchanged.
#include <algorithm>

#include "lp_kernel.cuh"

namespace lp {

// Squared distance from p to the triangle (a, a + ab, a + ac): closest point by Voronoi
// regions of the vertices, edges and face (Ericson, Real-Time Collision Detection, 2005).
__device__ __forceinline__ float point_triangle_dist2(V3 p, V3 a, V3 ab, V3 ac)
{
    const V3 ap = sub3(p, a);
    const float d1 = dot3(ab, ap), d2 = dot3(ac, ap);
    V3 q;
    if (d1 <= 0.0f && d2 <= 0.0f) {
        q = a;
    } else {
        const V3 b = add3(a, ab), c = add3(a, ac);
        const V3 bp = sub3(p, b);
        const float d3 = dot3(ab, bp), d4 = dot3(ac, bp);
        const V3 cp = sub3(p, c);
        const float d5 = dot3(ab, cp), d6 = dot3(ac, cp);
        const float vc = d1 * d4 - d3 * d2, vb = d5 * d2 - d1 * d6, va = d3 * d6 - d5 * d4;
        if (d3 >= 0.0f && d4 <= d3) {
            q = b;
        } else if (vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f) {
            q = add3(a, scl3(d1 / (d1 - d3), ab));
        } else if (d6 >= 0.0f && d5 <= d6) {
            q = c;
        } else if (vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f) {
            q = add3(a, scl3(d2 / (d2 - d6), ac));
        } else if (va <= 0.0f && (d4 - d3) >= 0.0f && (d5 - d6) >= 0.0f) {
            const float w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
            q = add3(b, scl3(w, sub3(c, b)));
        } else {
            const float den = 1.0f / (va + vb + vc);
            q = add3(a, add3(scl3(vb * den, ab), scl3(vc * den, ac)));
        }
    }
    const V3 d = sub3(p, q);
    return dot3(d, d);
}

__device__ __forceinline__ float box_dist2(float lo_x, float hi_x, float lo_y, float hi_y, float lo_z, float hi_z,
                                           V3 p)
{
    const float dx = fmaxf(fmaxf(lo_x - p.x, 0.0f), p.x - hi_x);
    const float dy = fmaxf(fmaxf(lo_y - p.y, 0.0f), p.y - hi_y);
    const float dz = fmaxf(fmaxf(lo_z - p.z, 0.0f), p.z - hi_z);
    return dx * dx + dy * dy + dz * dz;
}

// Distance^2 from p to the nearest triangle, or cap2 if none is closer.
__device__ float nearest_dist2(const KParams &P, V3 p, float cap2)
{
    float best = cap2;
    int stack[kStackDepth];
    int sp = 0, node = 0;
    for (;;) {
        const float4 a = __ldg(P.node_a + node), b = __ldg(P.node_b + node), c = __ldg(P.node_c + node);
        const int4 d = __ldg(P.node_d + node);
        const float d0 = box_dist2(a.x, a.y, a.z, a.w, c.x, c.y, p);
        const float d1 = box_dist2(b.x, b.y, b.z, b.w, c.z, c.w, p);
        int next[2];
        float nd[2];
        int k = 0;
        const int ref[2] = {d.x, d.y};
        const float dd[2] = {d0, d1};
        for (int s = 0; s < 2; ++s) {
            if (!(dd[s] < best)) continue;
            if (ref[s] < 0) {
                const int e = ~ref[s], f = e >> 3, cnt = (e & 7) + 1;
                for (int j = f; j < f + cnt; ++j) {
                    const float4 ta = __ldg(P.tri_a + j), tb = __ldg(P.tri_b + j), tc = __ldg(P.tri_c + j);
                    const float q = point_triangle_dist2(p, v3(ta.x, ta.y, ta.z), v3(ta.w, tb.x, tb.y),
                                                         v3(tb.z, tb.w, tc.x));
                    best = fminf(best, q);
                }
            } else {
                next[k] = ref[s];
                nd[k] = dd[s];
                ++k;
            }
        }
        if (k == 2) {
            const bool f0 = nd[0] <= nd[1];
            if (sp < kStackDepth) stack[sp++] = f0 ? next[1] : next[0];
            node = f0 ? next[0] : next[1];
        } else if (k == 1) {
            node = next[0];
        } else {
            // pop, skipping subtrees that the shrinking best has ruled out is left to the child test
            if (sp == 0) break;
            node = stack[--sp];
        }
    }
    return best;
}

// Safety grid, built level by level from blocks of 2^L x 2^L x 2^L cells (edge s = 2^L h)
// down to single cells.  A block's centre lies off = sqrt(3)/2 s from the centre of its
// parent block, so with dp the parent's distance, its own distance to the nearest
// triangle lies in [dp - off, dp + off] (the code widens both ends for rounding):
//  * lower end above near_T: the block is far from every triangle, and the lower end
//    is kept as its (conservative) distance, with no search;
//  * otherwise: a nearest-triangle search starting from the upper end, which prunes all
//    but the triangles around the block.
// near_T grows with the level so that the children of a far block are far too, and a
// near block's distance is always exact (capped at cap), as its children's upper end
// needs.  The top level has no parent and searches from cap.  Level 0 (Final) turns the
// cell-centre distance d into the cell's bound, in units of g_unit:
// (d - half_diag - eps) * 0.9999, rounded down.  eps covers the few-ulp overreach of the
// ray/triangle test; every value is a lower bound of the true distance.
template <bool Final>
__global__ void __launch_bounds__(256) safety_level_kernel(const __grid_constant__ KParams P, float s, int nx, int ny,
                                                           int nz, const float *parent, float off, float near_t,
                                                           float cap, float half_diag, float eps, float *dist,
                                                           uint16_t *out)
{
    const int64_t n = (int64_t)nx * ny * nz;
    const int px = (nx + 1) / 2, py = (ny + 1) / 2;
    const float tol = 1e-3f * P.g_unit * 256.0f;   // 1e-3 of a cell
    const float cap2 = cap * cap;
    const float inv_unit = 1.0f / P.g_unit;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int ix = (int)(i % nx);
        const int iy = (int)((i / nx) % ny);
        const int iz = (int)(i / ((int64_t)nx * ny));
        const V3 c = v3(P.g_ox + (ix + 0.5f) * s, P.g_oy + (iy + 0.5f) * s, P.g_oz + (iz + 0.5f) * s);
        float d;
        if (parent) {
            const float dp = parent[((int64_t)(iz >> 1) * py + (iy >> 1)) * px + (ix >> 1)];
            const float lb = (dp - off) * (1.0f - 1e-5f) - tol;
            if (lb > near_t) {
                d = lb;
            } else {
                const float r = fminf((dp + off) * (1.0f + 1e-5f) + tol, cap);
                float best2 = nearest_dist2(P, c, r * r);
                if (!(best2 < r * r) && r < cap) best2 = nearest_dist2(P, c, cap2);   // not reached
                d = sqrtf(best2);
            }
        } else {
            d = sqrtf(nearest_dist2(P, c, cap2));
        }
        if (Final) {
            const float safe = (d - half_diag - eps) * 0.9999f;
            const float q = safe > 0.0f ? floorf(safe * inv_unit) : 0.0f;
            out[i] = (uint16_t)fminf(q, 65535.0f);
        } else {
            dist[i] = d;
        }
    }
}

cudaError_t launch_safety_grid(const KParams &P, float h, float half_diag, float eps, float cap, float *const *levels,
                               int n_levels, uint16_t *out, cudaStream_t s)
{
    // thresholds: near_t[L + 1] >= near_t[L] + off[L] + margins, so far parents have far children
    float near_t[8], off[8];
    near_t[0] = 16.0f * h;
    for (int L = 0; L < n_levels; ++L) {
        off[L] = 0.8660254f * h * (float)(1 << L);
        near_t[L + 1] = near_t[L] * 1.0001f + off[L] + 0.01f * h;
    }
    for (int L = n_levels; L >= 0; --L) {
        const int nx = (P.g_nx + (1 << L) - 1) >> L, ny = (P.g_ny + (1 << L) - 1) >> L;
        const int nz = (P.g_nz + (1 << L) - 1) >> L;
        const int64_t n = (int64_t)nx * ny * nz;
        const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 16));
        const float *par = L < n_levels ? levels[L + 1] : nullptr;
        const float o = L < n_levels ? off[L] : 0.0f;
        if (L == 0)
            safety_level_kernel<true><<<grid, 256, 0, s>>>(P, h, nx, ny, nz, par, o, near_t[0], cap, half_diag, eps,
                                                            nullptr, out);
        else
            safety_level_kernel<false><<<grid, 256, 0, s>>>(P, h * (float)(1 << L), nx, ny, nz, par, o, near_t[L], cap,
                                                             half_diag, eps, levels[L], nullptr);
    }
    return cudaGetLastError();
}

// Triangle / cube overlap by the separating-axis theorem: the cube c +- r and the
// triangle (a, b, d) are disjoint iff their projections are disjoint on one of 13
// axes: the 3 cube axes, the triangle normal, and the 9 cross products of a cube axis
// with a triangle edge (Akenine-Moller, "Fast 3D triangle-box overlap testing", 2001).
// r includes a margin far above the rounding of the projections, so the test never
// reports "disjoint" for a triangle that touches the cube.
__device__ bool tri_cube_overlap(V3 c, float r, V3 a, V3 b, V3 d)
{
    const V3 v0 = sub3(a, c), v1 = sub3(b, c), v2 = sub3(d, c);
    if (fminf(v0.x, fminf(v1.x, v2.x)) > r || fmaxf(v0.x, fmaxf(v1.x, v2.x)) < -r) return false;
    if (fminf(v0.y, fminf(v1.y, v2.y)) > r || fmaxf(v0.y, fmaxf(v1.y, v2.y)) < -r) return false;
    if (fminf(v0.z, fminf(v1.z, v2.z)) > r || fmaxf(v0.z, fmaxf(v1.z, v2.z)) < -r) return false;
    const V3 e[3] = {sub3(v1, v0), sub3(v2, v1), sub3(v0, v2)};
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const V3 f = e[i];
        // axis x cross f = (0, -f.z, f.y)
        float p0 = f.y * v0.z - f.z * v0.y, p1 = f.y * v1.z - f.z * v1.y, p2 = f.y * v2.z - f.z * v2.y;
        float rr = r * (fabsf(f.y) + fabsf(f.z));
        if (fminf(p0, fminf(p1, p2)) > rr || fmaxf(p0, fmaxf(p1, p2)) < -rr) return false;
        // axis y cross f = (f.z, 0, -f.x)
        p0 = f.z * v0.x - f.x * v0.z; p1 = f.z * v1.x - f.x * v1.z; p2 = f.z * v2.x - f.x * v2.z;
        rr = r * (fabsf(f.x) + fabsf(f.z));
        if (fminf(p0, fminf(p1, p2)) > rr || fmaxf(p0, fmaxf(p1, p2)) < -rr) return false;
        // axis z cross f = (-f.y, f.x, 0)
        p0 = f.x * v0.y - f.y * v0.x; p1 = f.x * v1.y - f.y * v1.x; p2 = f.x * v2.y - f.y * v2.x;
        rr = r * (fabsf(f.x) + fabsf(f.y));
        if (fminf(p0, fminf(p1, p2)) > rr || fmaxf(p0, fmaxf(p1, p2)) < -rr) return false;
    }
    const V3 n = cross3(e[0], e[1]);
    return fabsf(dot3(n, v0)) <= r * (fabsf(n.x) + fabsf(n.y) + fabsf(n.z));
}

// One pass over the triangles (BVH order): every cell that a triangle touches (cells
// widened by eps) gets a count (refs == nullptr) or, in the second pass, the triangle's
// index at start[cell] + the next free slot (count re-zeroed before that pass).  One warp
// per triangle, its lanes striding over the cells of the triangle's box: a large
// triangle (a slab face covers 10^5 cells) is not left to a single thread.  The order of
// the entries within a cell is not defined, and no query depends on it.
__global__ void __launch_bounds__(256) cell_lists_kernel(const __grid_constant__ KParams P, int n_tri, float h,
                                                         float eps, uint32_t *count, const uint32_t *start,
                                                         int32_t *refs)
{
    const int lane = threadIdx.x & 31;
    const int n_warps = (gridDim.x * blockDim.x) >> 5;
    for (int j = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; j < n_tri; j += n_warps) {
        const float4 ta = __ldg(P.tri_a + j), tb = __ldg(P.tri_b + j), tc = __ldg(P.tri_c + j);
        const V3 a = v3(ta.x, ta.y, ta.z);
        const V3 b = add3(a, v3(ta.w, tb.x, tb.y)), d = add3(a, v3(tb.z, tb.w, tc.x));
        const float lo[3] = {fminf(a.x, fminf(b.x, d.x)), fminf(a.y, fminf(b.y, d.y)), fminf(a.z, fminf(b.z, d.z))};
        const float hi[3] = {fmaxf(a.x, fmaxf(b.x, d.x)), fmaxf(a.y, fmaxf(b.y, d.y)), fmaxf(a.z, fmaxf(b.z, d.z))};
        const float o[3] = {P.g_ox, P.g_oy, P.g_oz};
        const int n[3] = {P.g_nx, P.g_ny, P.g_nz};
        int c0[3], c1[3];
        for (int k = 0; k < 3; ++k) {
            c0[k] = min(max((int)floorf((lo[k] - eps - o[k]) * P.g_inv_h), 0), n[k] - 1);
            c1[k] = min(max((int)floorf((hi[k] + eps - o[k]) * P.g_inv_h), 0), n[k] - 1);
        }
        const int ex = c1[0] - c0[0] + 1, ey = c1[1] - c0[1] + 1;
        const int64_t n_cells = (int64_t)ex * ey * (c1[2] - c0[2] + 1);
        for (int64_t q = lane; q < n_cells; q += 32) {
            const int x = c0[0] + (int)(q % ex);
            const int y = c0[1] + (int)((q / ex) % ey);
            const int z = c0[2] + (int)(q / ((int64_t)ex * ey));
            const V3 c = v3(o[0] + ((float)x + 0.5f) * h, o[1] + ((float)y + 0.5f) * h, o[2] + ((float)z + 0.5f) * h);
            if (!tri_cube_overlap(c, 0.5f * h + eps, a, b, d)) continue;
            const int64_t cell = ((int64_t)z * n[1] + y) * n[0] + x;
            const uint32_t k = atomicAdd(count + cell, 1u);
            if (refs) refs[start[cell] + k] = j;
        }
    }
}

// Cell words from the safety bounds and the list layout (see KParams::cell_word).
// lists == false: every cell carries its safety bound only.
__global__ void cell_word_kernel(int64_t n, const uint16_t *safe, const uint32_t *count, const uint32_t *start,
                                 bool lists, uint32_t *word)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t k = lists ? count[i] : 0u;
        uint32_t w;
        if (k == 0) w = kCellEmpty | safe[i];
        else if (k >= kCellDense || start[i] + k > 0xffffffu) w = kCellDense << 24;
        else w = start[i] | (k << 24);
        word[i] = w;
    }
}

cudaError_t launch_cell_lists(const KParams &P, int n_tri, float h, float eps, uint32_t *count, const uint32_t *start,
                              int32_t *refs, cudaStream_t s)
{
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(((int64_t)n_tri * 32 + 255) / 256, 148 * 16));
    cell_lists_kernel<<<grid, 256, 0, s>>>(P, n_tri, h, eps, count, start, refs);
    return cudaGetLastError();
}

cudaError_t launch_cell_words(int64_t n, const uint16_t *safe, const uint32_t *count, const uint32_t *start, bool lists,
                              uint32_t *word, cudaStream_t s)
{
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 16));
    cell_word_kernel<<<grid, 256, 0, s>>>(n, safe, count, start, lists, word);
    return cudaGetLastError();
}

}  // namespace lp
