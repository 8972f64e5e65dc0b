// lp_transport_impl.cuh -- persistent photon-transport kernel for sm_100a.
//
// One CUDA thread carries one photon packet at a time, as one OpenCL work-item does
// in the reference (src/Simulation/MCLightPropagation.cl:1262-1606).  The grid is
// persistent: each warp refills the lanes whose photon has finished with new photon
// ids taken from a global counter, one atomicAdd per warp refill, so lanes stay busy
// until the photon budget is spent.  Photon i draws its random numbers from Philox
// blocks (key = seed, counter = (i, event, stream)), so results do not depend on
// which thread traced which photon; every loop iteration computes exactly one block,
// which keeps the warp converged on the RNG.
//
// Per loop iteration (MCLightPropagation.cl:1375-1575):
//   step length (.cl:1405-1442) -> nearest triangle within the step through the BVH
//   (replaces the O(T) FindTriangleInPath, .cl:1037-1093) -> boundary
//   (TransmitOrReflect, .cl:921-1018) or absorb + Henyey-Greenstein scatter +
//   absorption tallies (.cl:1513-1537) -> roulette (.cl:1539-1545).
// At the end of a photon its exit record (.cl:1583-1594) is binned on the device into
// the reference's SFT and RTd images (CalculatePropagation.cpp:1553-1626).
//
// Exact = true  keeps the reference's arithmetic operation by operation (compiled
//               with --fmad=false): a photon follows the oracle's trajectory for the
//               same random numbers up to last-place differences of logf/cosf/acosf.
// Exact = false (production) computes the same physics with fewer operations:
//               Henyey-Greenstein sampling with precomputed factors, the direction-
//               cosine update of Wang et al. (MCML, 1995) instead of two Rodrigues
//               rotations (same distribution: polar angle from HG, uniform azimuth),
//               vector refraction/reflection, reciprocal multiplies, explicit fused
//               multiply-adds.  No unit lets the compiler contract on its own, so a
//               device function gives the same bits in every kernel that inlines it.
#pragma once
#include <algorithm>

#include "lp_kernel.cuh"

namespace lp {

constexpr int kBlock = 256;
// Resident blocks per SM the single-instance kernel is compiled for (register budget
// 65536 / (kBlock x this)); the batched kernel's configurations are autotuned instead.
#ifndef LP_TRANSPORT_MIN_BLOCKS
#define LP_TRANSPORT_MIN_BLOCKS 3
#endif

struct Photon {
    float px, py, pz, vx, vy, vz;
    float w, unfin, absorbed;
    int32_t last_tri;        // face of the last boundary event, -1 before any: its normal is
                             // CalcAlphaOut's (.cl:1583), see photon_normal
    float exit_w;            // exit weight once scored
    int32_t curr, refTri;
    uint32_t steps;
    uint32_t flags;          // see F_*, EXIT_SHIFT, AXIS_SHIFT
    unsigned long long region_acc;
    uint32_t idx;            // photon index within the launch: the photon id is P.first + idx
    float seg_len;           // differentiation: path length and interactions in the
    uint32_t seg_k;          // current region since the photon entered it
    float safe;              // lower bound of the distance from the position to any triangle
};

// Per-photon, per-region path lengths and interaction counts of a differentiated run
// (thread-local, indexed by region id).
struct GradAcc {
    float L[kGradRegions];
    uint32_t k[kGradRegions];
};
// flags: bit 0 traversedFetalTissue, bit 1 roulette, bits 2-3 exit kind, bits 4-5 the
// on-axis normal override at the last boundary (0 none, 1 +eZ, 2 -eZ, 3 zero vector)
enum : uint32_t { F_FETAL = 1u, F_ROULETTE = 2u, EXIT_SHIFT = 2, AXIS_SHIFT = 4 };
enum : uint32_t { EXIT_NONE = 0, EXIT_SURF = 1, EXIT_SURF_FETAL = 2, EXIT_TRANS = 3 };

struct Counters {
    uint32_t scatter, boundary, query, roulette, rz_drop, vox_drop, skip, bvh;
};

template <bool Exact>
__device__ __forceinline__ float hg_cos_theta(const Medium &m, float xi)
{
    float cosTheta;
    if (Exact) {
        // VScatter (.cl:625-634)
        const float g = m.g;
        const float g1 = (1.0f - g * g) / (1.0f - g + 2.0f * g * xi);
        if (g != 0.0f) cosTheta = (1.0f + g * g - g1 * g1) / (2.0f * g);
        else cosTheta = 2.0f * xi - 1.0f;
    } else {
        if (m.g != 0.0f) {
            const float g1 = __fdividef(m.hg_a, __fmaf_rn(m.hg_c, xi, m.hg_b));
            cosTheta = __fmaf_rn(-g1, g1, m.hg_d) * m.hg_inv2g;
        } else {
            cosTheta = __fmaf_rn(2.0f, xi, -1.0f);
        }
    }
    return fminf(fmaxf(cosTheta, -1.0f), 1.0f);
}

// Rotate (.cl:697-708)
__device__ __forceinline__ V3 rotate(V3 vec, V3 axis, float c, float s)
{
    const float nDx = dot3(axis, vec);
    const V3 nXx = cross3(axis, vec);
    const V3 nXxXn = cross3(nXx, axis);
    return add3(add3(scl3(nDx, axis), scl3(c, nXxXn)), scl3(s, nXx));
}

__device__ __forceinline__ V3 fast_norm(V3 v)
{
    const float r = rsqrtf(__fmaf_rn(v.x, v.x, __fmaf_rn(v.y, v.y, v.z * v.z)));
    return v3(v.x * r, v.y * r, v.z * r);
}

template <bool Exact>
__device__ __forceinline__ V3 scatter_direction(V3 v, const Medium &m, float xt, float xp)
{
    const float cosTheta = hg_cos_theta<Exact>(m, xt);
    if (Exact) {
        // VScatter (.cl:597-655): rotate by theta about e_rot _|_ v, then by psi about v
        V3 e_rot = v3(0.0f, 0.0f, 0.0f);
        if (v.z != 0.0f) {
            const float z = -(v.x + v.y) / (v.z);
            e_rot = v3(1.0f, 1.0f, z);
        } else if (v.y != 0.0f) {
            const float y = -(v.x) / (v.y);
            e_rot = v3(1.0f, y, 0.0f);
        } else if (v.x != 0.0f) {
            e_rot = v3(0.0f, 1.0f, 0.0f);
        }
        e_rot = norm3(e_rot);
        const float sinTheta = sqrtf(1.0f - cosTheta * cosTheta);
        const float psi = 2.0f * 3.14159265358979323846f * xp;
        const float cosPsi = cosf(psi);
        float sinPsi = sqrtf(1.0f - cosPsi * cosPsi);
        if (psi > 3.14159265358979323846f) sinPsi *= -1.0f;
        const V3 rot_theta = norm3(rotate(v, e_rot, cosTheta, sinTheta));
        return norm3(rotate(rot_theta, v, cosPsi, sinPsi));
    } else {
        // direction-cosine update (Wang, Jacques & Zheng, MCML 1995).  1 - uz^2 is taken
        // as ux^2 + uy^2 (|v| = 1), which keeps its precision near the z axis where the
        // difference form cancels; the axial case scatters about z with uz' = sign(uz) cos.
        const float sinTheta = sqrtf(fmaxf(0.0f, __fmaf_rn(-cosTheta, cosTheta, 1.0f)));
        float sinPsi, cosPsi;
        sincospif(2.0f * xp, &sinPsi, &cosPsi);
        V3 r;
        const float uz2 = __fmaf_rn(v.x, v.x, v.y * v.y);
        if (uz2 < 1e-20f) {
            r = v3(sinTheta * cosPsi, sinTheta * sinPsi, v.z > 0.0f ? cosTheta : -cosTheta);
        } else {
            const float it = rsqrtf(uz2);
            const float temp = uz2 * it;  // sqrt(1 - uz^2)
            const float st = sinTheta * it;
            r = v3(__fmaf_rn(st, __fmaf_rn(v.x * v.z, cosPsi, -v.y * sinPsi), v.x * cosTheta),
                   __fmaf_rn(st, __fmaf_rn(v.y * v.z, cosPsi, v.x * sinPsi), v.y * cosTheta),
                   __fmaf_rn(-sinTheta * cosPsi, temp, v.z * cosTheta));
        }
        return fast_norm(r);
    }
}

// GetFresnel (.cl:857-907)
__device__ __forceinline__ float fresnel(float n1, float n2, float cosIn)
{
    float r;
    if (n1 == n2) {
        r = 0.0f;
    } else if (fabsf(cosIn) == 1.0f) {
        r = (n1 - n2) / (n1 + n2);
        r *= r;
    } else if (cosIn == 0.0f) {
        r = 1.0f;
    } else {
        const float sinIn = sqrtf(1.0f - cosIn * cosIn);
        const float sinOut = n1 * sinIn / n2;
        if (sinOut >= 1.0f) {
            r = 1.0f;
        } else {
            const float cosOut = sqrtf(1.0f - sinOut * sinOut);
            const float cap = cosIn * cosOut - sinIn * sinOut;
            const float cam = cosIn * cosOut + sinIn * sinOut;
            const float sap = sinIn * cosOut + cosIn * sinOut;
            const float sam = sinIn * cosOut - cosIn * sinOut;
            r = 0.5f * (sam * sam) * ((cam * cam) + (cap * cap)) / ((sap * sap) * (cam * cam));
        }
    }
    return r;
}

// Sum of x over the lanes of grp (a __match_any_sync group, every lane of it calling),
// exact for x < 2^59: the three slices x[0:16], x[16:32], x[32:64] are reduced by
// redux.sync, and each slice's sum over at most 32 lanes fits in 32 bits.
__device__ __forceinline__ unsigned long long group_sum_u64(unsigned grp, unsigned long long x)
{
    const unsigned a = __reduce_add_sync(grp, (unsigned)(x & 0xffffull));
    const unsigned b = __reduce_add_sync(grp, (unsigned)((x >> 16) & 0xffffull));
    const unsigned c = __reduce_add_sync(grp, (unsigned)(x >> 32));
    return (unsigned long long)a + ((unsigned long long)b << 16) + ((unsigned long long)c << 32);
}

__device__ __forceinline__ void add_fix(unsigned long long *a, float w)
{
    const unsigned long long f = fix32(w);
    if (f) atomicAdd(a, f);
}

// Differentiation: the photon scored surface weight s in ring d.  With path density
// prod_r mus_r^k_r exp(-(mua_r + mus_r) L_r / factor) times the albedo weights, the
// score's derivatives are s * (-L_r / factor) for mua_r and s * (k_r / mus_r - L_r / factor)
// for mus_r (perturbation Monte Carlo, Hayakawa et al., Opt. Lett. 26, 2001); the
// kernel accumulates the moments of s L_r and s k_r, the host forms the derivatives.
static __device__ __noinline__ void score_gradient(const KParams &P, const GradAcc &ga, int d, float s)
{
    double *g = P.grad + 5 * (int64_t)d * P.n_media;
    for (int r = 0; r < P.n_media; ++r) {
        const double a = (double)s * (double)ga.L[r];
        const double b = (double)s * (double)ga.k[r];
        if (a == 0.0 && b == 0.0) continue;
        atomicAdd(g + 5 * r + 0, a);
        atomicAdd(g + 5 * r + 1, b);
        atomicAdd(g + 5 * r + 2, a * a);
        atomicAdd(g + 5 * r + 3, b * b);
        atomicAdd(g + 5 * r + 4, a * b);
    }
}

// The normal of the photon's last boundary event as the transport used it: the face's unit
// normal, the on-axis override (sign * eZ), or (0, 0, -1) before any event (PhotonClass
// init, .cl:344-389).  Kept as the face index and two flag bits instead of three floats.
__device__ __forceinline__ V3 photon_normal(const KParams &P, const Photon &ph)
{
    const uint32_t axis = (ph.flags >> AXIS_SHIFT) & 3u;
    if (axis) {
        const float sg = axis == 1u ? 1.0f : (axis == 2u ? -1.0f : 0.0f);
        return scl3(sg, v3(P.nzx, P.nzy, P.nzz));
    }
    if (ph.last_tri < 0) return v3(0.0f, 0.0f, -1.0f);
    const float4 at = __ldg(P.tri_attr + ph.last_tri);
    return v3(at.x, at.y, at.z);
}

// Exit record binning of CalculatePropagation.cpp:1553-1626 plus radial bins and rings.
template <bool Grad>
static __device__ __noinline__ void finish_photon(const KParams &P, const Photon &ph, const GradAcc *ga)
{
    const V3 v = v3(ph.vx, ph.vy, ph.vz), nv = photon_normal(P, ph);
    const float alpha = fabsf(acosf(dot3(v, nv)));
    const V3 d = v3(P.poix - ph.px, P.poiy - ph.py, P.poiz - ph.pz);
    const float radius = sqrtf(d.x * d.x + d.y * d.y + d.z * d.z);
    const V3 pr = v3(ph.px - P.poix, ph.py - P.poiy, ph.pz - P.poiz);
    const float cx = dot3(v3(P.nxx, P.nxy, P.nxz), pr);
    const float cy = dot3(v3(P.nyx, P.nyy, P.nyz), pr);
    const float cz = dot3(v3(P.nzx, P.nzy, P.nzz), pr);
    const uint32_t kind = (ph.flags >> EXIT_SHIFT) & 3u;
    const float s = (kind == EXIT_SURF || kind == EXIT_SURF_FETAL) ? ph.exit_w : 0.0f;
    const float f = (kind == EXIT_SURF_FETAL) ? ph.exit_w : 0.0f;
    const float t = (kind == EXIT_TRANS) ? ph.exit_w : 0.0f;
    const int64_t slot = (int64_t)ph.idx;
    if (P.exit_rec && slot >= 0 && slot < P.exit_cap) {
        float4 *r = reinterpret_cast<float4 *>(P.exit_rec + 8 * slot);
        r[0] = make_float4(cx, cy, cz, s);
        r[1] = make_float4(f, t, alpha, radius);
    }
    if (kind == EXIT_NONE) return;
    int x = trunc_sat(cx / P.dg[0]);
    int y = trunc_sat(cy / P.dg[1]);
    y = min(max(y, -P.hy), P.hy);
    x = min(max(x, -P.hx), P.hx);
    unsigned long long *c = P.sft + 3 * ((int64_t)(y + P.hy) * P.sft_nx + (x + P.hx));
    add_fix(c + 0, s);
    add_fix(c + 1, f);
    add_fix(c + 2, t);
    int ai = trunc_sat_d(((double)(alpha * 180.0f) / 3.14159265358979323846) / (double)P.dg[5]);
    int ri = trunc_sat(radius / P.dg[3]);
    if (ri > P.dimR - 1) ri = P.dimR - 1;
    else if (ri < 0) ri = 0;
    if (ai > P.dimAlpha - 1) ai = P.dimAlpha - 1;
    else if (ai < 0) ai = 0;
    unsigned long long *r = P.rtd + 3 * ((int64_t)ai * P.dimR + ri);
    add_fix(r + 0, s);
    add_fix(r + 1, f);
    add_fix(r + 2, t);
    const float rho = sqrtf(cx * cx + cy * cy);
    if (P.n_rbins > 0) {
        const int b = trunc_sat(rho / P.rbin_dr);
        if (b >= 0 && b < P.n_rbins) {
            add_fix(P.rbins + 2 * b, s);
            add_fix(P.rbins + 2 * b + 1, t);
        }
    }
    if (s > 0.0f) {
        for (int k = 0; k < P.n_det; ++k) {
            if (rho >= P.det_lo[k] && rho < P.det_hi[k]) {
                add_fix(P.det + 2 * k, s);
                add_fix(P.det + 2 * k + 1, s * s);
                if (Grad) score_gradient(P, *ga, k, s);
            }
        }
    }
}

__device__ __forceinline__ void start_photon(const KParams &P, Photon &ph, uint32_t idx)
{
    const int64_t pid = P.first + (int64_t)idx;
    // PhotonClass::Init (.cl:344-389) with vStart[0] (.cl:429-467)
    ph.px = P.p0x; ph.py = P.p0y; ph.pz = P.p0z;
    ph.vx = P.v0x; ph.vy = P.v0y; ph.vz = P.v0z;
    if (P.src_type == 1) {
        // fibre source (no reference counterpart), event 0: disk of radius src_radius in
        // the (eX, eY) plane, direction uniform in solid angle within the cone about eZ
        EventRng rng;
        rng.draw((uint64_t)pid, 0u, P.stream, P.key0, P.key1);
        const V3 ex = v3(P.nxx, P.nxy, P.nxz), ey = v3(P.nyx, P.nyy, P.nyz), ez = v3(P.nzx, P.nzy, P.nzz);
        const float r = P.src_radius * sqrtf(rng.u0);
        const float phi = 2.0f * 3.14159265358979323846f * rng.u1;
        const float cp = cosf(phi), sp = sinf(phi);
        const V3 p = add3(v3(ph.px, ph.py, ph.pz), add3(scl3(r * cp, ex), scl3(r * sp, ey)));
        ph.px = p.x; ph.py = p.y; ph.pz = p.z;
        const float ct = 1.0f - rng.u2 * (1.0f - P.src_cos_max);
        const float stt = sqrtf(1.0f - ct * ct);
        const float psi = 2.0f * 3.14159265358979323846f * rng.u3;
        const float cq = cosf(psi), sq = sinf(psi);
        const V3 v = norm3(add3(scl3(ct, ez), add3(scl3(stt * cq, ex), scl3(stt * sq, ey))));
        ph.vx = v.x; ph.vy = v.y; ph.vz = v.z;
    }
    ph.w = P.w0;
    ph.unfin = 0.0f;
    ph.absorbed = 0.0f;
    ph.last_tri = -1;
    ph.exit_w = 0.0f;
    ph.curr = 0;
    ph.refTri = -1;
    ph.steps = 0;
    ph.flags = F_ROULETTE;
    ph.region_acc = 0;
    ph.idx = idx;
    ph.seg_len = 0.0f;
    ph.seg_k = 0;
    ph.safe = 0.0f;
}

// A boundary event (.cl:1443-1465 with TransmitOrReflect, .cl:921-1018): the photon moves
// thit to the face `tri` (-1: no face, it leaves the model), then is transmitted or
// reflected with probability from the Fresnel equations (xi against R).  Out of line: it
// runs about once per hundred steps, and keeping its code out of the step loop keeps the
// loop's instructions in cache for the warps that scatter.  The photon goes in and comes
// back by value: a reference would take its address out of the step loop, and the
// compiler would then keep the photon in local memory on every step.
template <bool Exact, bool Grad>
static __device__ __forceinline__ Photon boundary_event(const KParams &P, const Medium *s_media,
                                                     unsigned long long *s_region, unsigned long long *s_cnt,
                                                     Photon ph, GradAcc *ga, int tri, float thit, float step,
                                                     float xi)
{
    [[maybe_unused]] unsigned long long *const dbg = P.counters ? P.counters + kBoundsCounter : nullptr;
    const Medium m = s_media[ph.curr];
    const V3 v = v3(ph.vx, ph.vy, ph.vz);
    ph.safe = 0.0f;
    ph.px = ph.px + thit * ph.vx;
    ph.py = ph.py + thit * ph.vy;
    ph.pz = ph.pz + thit * ph.vz;
    ph.refTri = -1;
    if (tri < 0) {
        // the reference would read mediumIDs[-1] here; the photon leaves the model
        atomicAdd(s_cnt + 4, 1ull);
        ph.w = 0.0f;
    } else if (LP_IN_RANGE(dbg, tri, P.n_tri)) {
        const float4 at = __ldg(P.tri_attr + tri);
        const int ids = __float_as_int(at.w);
        const int inner = ids & 0xffff, outer = ids >> 16;
        V3 nv = v3(at.x, at.y, at.z);
        int nxt_id = (ph.curr == outer) ? inner : outer;
        // a photon whose region is neither side of the face it meets has passed through
        // another face unseen (a crack between triangles that the float test leaves)
        if (ph.curr != inner && ph.curr != outer) atomicAdd(s_cnt + 14, 1ull);
        if (!LP_IN_RANGE(dbg, nxt_id, P.n_media)) nxt_id = ph.curr;
        const Medium nx = s_media[nxt_id];
        uint32_t axis = 0u;
        if (P.compat & 0x2u) {
            if (fabsf(sqrtf(ph.px * ph.px + ph.py * ph.py)) < 0.01f) {
                const float sg = sign_cl(dot3(nv, v3(P.ezx, P.ezy, P.ezz)));
                nv = scl3(sg, v3(P.nzx, P.nzy, P.nzz));
                axis = sg > 0.0f ? 1u : (sg < 0.0f ? 2u : 3u);
            }
        }
        ph.last_tri = tri;
        ph.flags = (ph.flags & ~(3u << AXIS_SHIFT)) | (axis << AXIS_SHIFT);
        // TransmitOrReflect (.cl:921-1018)
        const float cosIn = dot3(nv, v);
        const float absCosIn = fabsf(cosIn);
        const float n1 = m.n, n2 = nx.n;
        float cos_crit = 0.0f;
        if (n1 > n2) cos_crit = sqrtf(1.0f - (n2 / n1) * (n2 / n1));
        float r;
        if (absCosIn <= cos_crit) r = 1.0f;
        else r = fresnel(n1, n2, (P.compat & 0x4u) ? cosIn : absCosIn);
        int newID;
        float muaNew, musNew;
        V3 vout;
        if (Exact) {
            const V3 e_y = norm3(cross3(nv, cross3(nv, v)));
            if (xi > r) {
                const float sinT = sqrtf(1.0f - cosIn * cosIn) * n1 / n2;
                float cosT = -sqrtf(1.0f - sinT * sinT);
                if (cosIn > 0.0f) cosT = fabsf(cosT);
                vout = norm3(sub3(scl3(cosT, nv), scl3(sinT, e_y)));
            } else {
                const float sinR = sqrtf(1.0f - cosIn * cosIn);
                const V3 t = norm3(add3(scl3(cosIn, nv), scl3(sinR, e_y)));
                vout = v3(-t.x, -t.y, -t.z);
            }
        } else {
            if (xi > r) {
                // v' = cosT n - sinT e_y with e_y = (n cosIn - v) / sinIn (unit n, v)
                const float s2 = fmaxf(0.0f, 1.0f - cosIn * cosIn);
                const float sinT = sqrtf(s2) * __fdividef(n1, n2);
                float cosT = sqrtf(fmaxf(0.0f, 1.0f - sinT * sinT));
                if (!(cosIn > 0.0f)) cosT = -cosT;
                const float k = s2 > 1e-12f ? sinT * rsqrtf(s2) : 0.0f;
                vout = fast_norm(v3(cosT * nv.x - k * (nv.x * cosIn - v.x), cosT * nv.y - k * (nv.y * cosIn - v.y),
                                    cosT * nv.z - k * (nv.z * cosIn - v.z)));
            } else {
                vout = fast_norm(v3(v.x - 2.0f * cosIn * nv.x, v.y - 2.0f * cosIn * nv.y,
                                    v.z - 2.0f * cosIn * nv.z));
            }
        }
        if (xi > r) {
            newID = (cosIn > 0.0f) ? outer : inner;
            muaNew = nx.mua;
            musNew = nx.mus;
        } else {
            newID = ph.curr;
            muaNew = m.mua;
            musNew = m.mus;
        }
        ph.vx = vout.x; ph.vy = vout.y; ph.vz = vout.z;
        if (!Exact) {
            // The hit point lies on the face's plane only to float rounding, on either
            // side.  On the wrong side, the next segment can cross a neighbouring face of
            // the same surface a rounding distance away (the face itself is excluded by
            // refTri): a spurious second boundary event, which in float happens to about
            // 2e-4 of the photons of a curved mesh and lets them leave the region they
            // are labelled with.  The production arithmetic moves the photon off the
            // plane, to the side it travels to, by a few rounding units of the scene's
            // coordinates and of the distance travelled.  (The reference-order
            // arithmetic keeps the reference's behaviour.)
            const float push = P.boundary_push + 1e-6f * thit;
            const float sp = (dot3(vout, nv) > 0.0f) ? push : -push;
            ph.px = __fmaf_rn(sp, nv.x, ph.px);
            ph.py = __fmaf_rn(sp, nv.y, ph.py);
            ph.pz = __fmaf_rn(sp, nv.z, ph.pz);
        }
        if (muaNew == 0.0f || musNew == 0.0f) {
            const float dist = fabsf(dot3(v3(P.nzx, P.nzy, P.nzz),
                                          v3(ph.px - P.poix, ph.py - P.poiy, ph.pz - P.poiz)));
            uint32_t kind;
            if (dist > P.distMin) kind = EXIT_TRANS;
            else kind = (ph.flags & F_FETAL) ? EXIT_SURF_FETAL : EXIT_SURF;
            ph.exit_w = ph.w * P.exitScale;
            ph.flags = (ph.flags & ~(3u << EXIT_SHIFT)) | (kind << EXIT_SHIFT);
            ph.w = 0.0f;
        }
        const int prev = ph.curr;
        ph.curr = newID;
        ph.refTri = tri;
        if (newID == P.fetal_id) ph.flags |= F_FETAL;
        ph.unfin = Exact ? (step - thit) * m.mut : fmaxf(step - thit, 0.0f) * m.mut;
        if (newID != prev) {
            if (ph.region_acc) atomicAdd(s_region + prev, ph.region_acc);
            ph.region_acc = 0;
            if (Grad) {
                ga->L[prev] += ph.seg_len + thit;
                ga->k[prev] += ph.seg_k;
                ph.seg_len = 0.0f;
                ph.seg_k = 0;
            }
        } else if (Grad) {
            ph.seg_len += thit;
        }
    } else {
        ph.w = 0.0f;   // debug build: a triangle index out of range ends the photon
    }
    return ph;
}

// A step in three parts: propose_step draws the event's random numbers and the step
// length and decides whether the step can reach a triangle; query_step finds the nearest
// triangle within reach; complete_step moves the photon (boundary event, or absorption and
// scattering), scores it and plays roulette.  One call of each in turn is one iteration of
// the reference's do-while loop (.cl:1388-1600).  (Letting the lanes whose step needs a
// query wait until several of a warp do, and running their queries together, measured
// slower on every batch size: the waiting lanes cost more steps per warp iteration than
// the shared queries save.)
struct Pending {
    float step, reach, safe_here;   // step length, its reach, distance bound at the position
    float u1, u2, u3;               // the event's uniforms after the step length's
    uint32_t word;                  // cell word at the position
};
enum : int { kStepEnded = 0, kStepClear = 1, kStepQuery = 2 };

// kStepQuery: the step may reach a triangle and needs a query; kStepClear: no triangle
// lies within its reach (complete_step with tri = -1); kStepEnded: the photon ended
// (debug build: a region id out of range).
template <bool Exact>
__device__ __forceinline__ int propose_step(const KParams &P, const Medium *s_media, Photon &ph, Counters &cnt,
                                            Pending &pd)
{
    // The cell word is read on every step, its load issued before the Philox rounds so
    // that they hide its latency (reading it only when the carried bound is used up saves
    // loads but waits on them: 1.3 % slower on the 660 nm abdomen).
    const uint32_t word = cell_at(P, ph.px, ph.py, ph.pz);
    EventRng rng;
    rng.draw((uint64_t)(P.first + (int64_t)ph.idx), ph.steps + 1u, P.stream, P.key0, P.key1);
    [[maybe_unused]] unsigned long long *const dbg = P.counters ? P.counters + kBoundsCounter : nullptr;
    if (!LP_IN_RANGE(dbg, ph.curr, P.n_media)) {
        ph.w = 0.0f;
        return kStepEnded;
    }
    const Medium m = s_media[ph.curr];
    float step = 0.0f;
    if (!m.ambient) {
        if (ph.unfin == 0.0f) {
            if (Exact) step = -logf(rng.u0) * P.factor / m.mut;
            else step = -logf(rng.u0) * P.factor * m.inv_mut;
        } else {
            step = Exact ? ph.unfin / m.mut : ph.unfin * m.inv_mut;
            ph.unfin = 0.0f;
        }
    }
    pd.step = step;
    // reach: the production arithmetic also takes a face that lies up to a few rounding
    // units beyond the step as the step's boundary.  A hit computed just past the step
    // although it lies just within it would otherwise let the photon end its step on the
    // far side of the face, outside the region it is labelled with.  The photon then stops
    // on the face (and is moved off it, see boundary_event) with no residual step.
    const float reach = Exact ? step : step + P.boundary_push + 1e-6f * step;
    pd.reach = reach;
    pd.u1 = rng.u1;
    pd.u2 = rng.u2;
    pd.u3 = rng.u3;
    // safe_here: lower bound of the distance from p to every triangle.  A step shorter
    // than it cannot reach one, so its bounded query would return "no hit" and is skipped;
    // after the step the bound shrinks by the step (plus the rounding of the move).
    pd.safe_here = ph.safe;
    pd.word = word;
    if (m.ambient) return kStepQuery;
    if (reach < pd.safe_here) {
        cnt.skip++;
        return kStepClear;
    }
    if (word & kCellEmpty) {
        // a cell no triangle touches: its word holds a bound for all its points (the
        // larger of two lower bounds is one too)
        pd.safe_here = fmaxf(pd.safe_here, safe_distance(P, word));
        if (reach < pd.safe_here) {
            cnt.skip++;
            return kStepClear;
        }
    }
    return kStepQuery;
}

// The nearest triangle within the step's reach (-1: none) and its distance thit; updates
// the distance bound the query establishes.
template <int STACK>
__device__ __forceinline__ int query_step(const KParams &P, const MeshView &M, const Medium *s_media,
                                          const Photon &ph, Counters &cnt, Pending &pd, float &thit)
{
    const V3 p = v3(ph.px, ph.py, ph.pz), v = v3(ph.vx, ph.vy, ph.vz);
    int tri = -1;
    if (s_media[ph.curr].ambient) {
        tri = query_nearest<STACK>(M, p, v, ph.refTri, kNoHit, thit);
        cnt.query++;
        cnt.bvh++;
        return tri;
    }
    // an empty cell: pd.safe_here holds its bound, which the step exceeds; a listed cell
    // raises it from the planes of its triangles when its list decides the step
    bool used_bvh;
    tri = grid_query<STACK>(P, M, p, v, ph.refTri, pd.reach, pd.word, thit, pd.safe_here, used_bvh);
    cnt.query++;
    cnt.bvh += used_bvh ? 1u : 0u;
    return tri;
}

// Returns false when the photon ends.  Agg: absorption deposits summed per cell across
// the warp before the atomic adds.
template <bool Exact, bool Grad, bool Agg = false>
__device__ __forceinline__ bool complete_step(const KParams &P, const Medium *s_media, unsigned long long *s_region,
                                              unsigned long long *s_cnt, Photon &ph, Counters &cnt, GradAcc *ga,
                                              const Pending &pd, int tri, float thit)
{
    const Medium m = s_media[ph.curr];
    const V3 v = v3(ph.vx, ph.vy, ph.vz);
    float step = pd.step;
    const float reach = pd.reach, safe_here = pd.safe_here;
    if (m.ambient) step = thit;
    const bool boundary = (tri >= 0) ? (thit <= (m.ambient ? step : reach)) : (kNoHit <= step);
    if (boundary) {
        cnt.boundary++;
        ph = boundary_event<Exact, Grad>(P, s_media, s_region, s_cnt, ph, Grad ? ga : nullptr, tri, thit, step, pd.u1);
    } else {
        cnt.scatter++;
        ph.px = ph.px + step * ph.vx;
        ph.py = ph.py + step * ph.vy;
        ph.pz = ph.pz + step * ph.vz;
        ph.refTri = -1;
        ph.safe = fmaxf(safe_here - step - P.step_eps, 0.0f);
        if (Grad) {
            ph.seg_len += step;
            ph.seg_k++;
        }
        if (m.absorbs) {
            ph.absorbed = ph.w * m.alb;
            ph.w -= ph.absorbed;
        }
        const V3 vn = scatter_direction<Exact>(v, m, pd.u1, pd.u2);
        ph.vx = vn.x; ph.vy = vn.y; ph.vz = vn.z;
        const V3 pr = v3(ph.px - P.poix, ph.py - P.poiy, ph.pz - P.poiz);
        const float cx = dot3(v3(P.nxx, P.nxy, P.nxz), pr);
        const float cy = dot3(v3(P.nyx, P.nyy, P.nyz), pr);
        const float cz = dot3(v3(P.nzx, P.nzy, P.nzz), pr);
        const float dw = ph.absorbed;
        const unsigned long long fdw = fix32(dw);
        // r-z grid (RecordAbsorbtionRZ, .cl:254-271, with atomic adds and z rows)
        int row, col;
        if (Exact) {
            const float rad = sqrtf(cx * cx + cy * cy) * sign_cl(cx) / P.dg[3];
            row = (int)floorf(cz / P.dg[2]);
            col = (int)floorf(rad + (float)P.dimR);
        } else {
            const float rad = copysignf(sqrtf(cx * cx + cy * cy), cx) * P.inv_dr;
            row = (int)floorf(cz * P.inv_dz);
            col = (int)floorf(rad + (float)P.dimR);
        }
        const bool rz_in = row >= 0 && row < P.rz_nz && col >= 0 && col < P.rz_nr;
        const unsigned long long fdm = (m.mua > 0.0f) ? fix32(Exact ? dw / m.mua : dw * m.inv_mua) : 0ull;
        int vox_key = -1;
        if (P.vox_nx > 0) {
            int ix, iy, iz;
            if (Exact) {
                ix = (int)floorf(cx / P.vox_dx + 0.5f * (float)P.vox_nx);
                iy = (int)floorf(cy / P.vox_dy + 0.5f * (float)P.vox_ny);
                iz = (int)floorf(cz / P.vox_dz);
            } else {
                ix = (int)floorf(cx * P.inv_vdx + 0.5f * (float)P.vox_nx);
                iy = (int)floorf(cy * P.inv_vdy + 0.5f * (float)P.vox_ny);
                iz = (int)floorf(cz * P.inv_vdz);
            }
            if (ix >= 0 && ix < P.vox_nx && iy >= 0 && iy < P.vox_ny && iz >= 0 && iz < P.vox_nz)
                vox_key = (iz * P.vox_ny + iy) * P.vox_nx + ix;
            else
                cnt.vox_drop++;
        }
        if (!rz_in) cnt.rz_drop++;
        const int rz_key = rz_in ? row * P.rz_nr + col : -1;
        if (Agg) {
            // warp-aggregated deposits: the lanes of this branch that hit the same cell
            // are matched, their fixed-point values summed exactly, and one leader per
            // cell issues the atomic add (integer sums: same tallies as the plain form)
            const unsigned lane = threadIdx.x & 31u;
            const unsigned act = __activemask();
            const unsigned g_rz = __match_any_sync(act, rz_key);
            if (rz_key >= 0) {
                const unsigned long long a = group_sum_u64(g_rz, fdw), b = group_sum_u64(g_rz, fdm);
                if (lane == (unsigned)(__ffs(g_rz) - 1)) {
                    unsigned long long *c = P.rz + 2 * (int64_t)rz_key;
                    if (a) atomicAdd(c, a);
                    if (b) atomicAdd(c + 1, b);
                    atomicAdd(s_cnt + 15, 1ull);   // leaders: 1 - leaders / deposits is the match rate
                }
            }
            const unsigned g_vox = __match_any_sync(act, vox_key);
            if (vox_key >= 0) {
                const unsigned long long a = group_sum_u64(g_vox, fdw);
                if (a && lane == (unsigned)(__ffs(g_vox) - 1)) atomicAdd(P.vox + vox_key, a);
            }
        } else {
            if (rz_key >= 0) {
                unsigned long long *c = P.rz + 2 * (int64_t)rz_key;
                if (fdw) atomicAdd(c, fdw);
                if (fdm) atomicAdd(c + 1, fdm);
            }
            if (vox_key >= 0 && fdw) atomicAdd(P.vox + vox_key, fdw);
        }
        ph.region_acc += fdw;
    }
    if (ph.w < P.w_th && ph.w > 0.0f) {
        cnt.roulette++;
        if (pd.u3 < P.chance) {
            ph.w /= P.chance;
            ph.flags |= F_ROULETTE;
        } else {
            ph.w = 0.0f;
            ph.flags &= ~F_ROULETTE;
        }
    }
    ph.steps++;
    if (P.max_steps > 0 && (int64_t)ph.steps >= P.max_steps && ph.w > 0.0f) {
        atomicAdd(s_cnt + 5, 1ull);
        ph.w = 0.0f;
    }
    return ph.w > 0.0f && (ph.w > P.w_th || (ph.flags & F_ROULETTE));
}

// One iteration of the reference's do-while loop, the three parts in turn.  Returns false
// when the photon ends.
template <bool Exact, bool Grad, int STACK = kStackDepth, bool Agg = false>
__device__ __forceinline__ bool step_photon(const KParams &P, const MeshView &M, const Medium *s_media,
                                            unsigned long long *s_region, unsigned long long *s_cnt,
                                            Photon &ph, Counters &cnt, GradAcc *ga)
{
    Pending pd;
    const int st = propose_step<Exact>(P, s_media, ph, cnt, pd);
    if (st == kStepEnded) return false;
    float thit = kNoHit;
    int tri = -1;
    if (st == kStepQuery) tri = query_step<STACK>(P, M, s_media, ph, cnt, pd, thit);
    return complete_step<Exact, Grad, Agg>(P, s_media, s_region, s_cnt, ph, cnt, ga, pd, tri, thit);
}

struct SmemLayout {
    int off_media, off_region, off_cnt, off_na, off_nb, off_nc, off_nd, off_ta, off_tb, off_tc, bytes;
};

__host__ __device__ inline SmemLayout smem_layout(int nodes_smem, int tris_smem)
{
    SmemLayout L;
    int o = 0;
    L.off_media = o; o += kMaxMedia * (int)sizeof(Medium);
    L.off_region = o; o += kMaxMedia * 8;
    L.off_cnt = o; o += 16 * 8;
    L.off_na = o; o += nodes_smem * 16;
    L.off_nb = o; o += nodes_smem * 16;
    L.off_nc = o; o += nodes_smem * 16;
    L.off_nd = o; o += nodes_smem * 16;
    L.off_ta = o; o += tris_smem * 16;
    L.off_tb = o; o += tris_smem * 16;
    L.off_tc = o; o += tris_smem * 16;
    L.bytes = o;
    return L;
}

__device__ __forceinline__ MeshView stage_mesh(const KParams &P, unsigned char *smem, const SmemLayout &L)
{
    MeshView M;
    M.na = P.node_a; M.nb = P.node_b; M.nc = P.node_c; M.nd = P.node_d;
    M.ta = P.tri_a; M.tb = P.tri_b; M.tc = P.tri_c;
    float4 *sa = reinterpret_cast<float4 *>(smem + L.off_na);
    float4 *sb = reinterpret_cast<float4 *>(smem + L.off_nb);
    float4 *sc = reinterpret_cast<float4 *>(smem + L.off_nc);
    int4 *sd = reinterpret_cast<int4 *>(smem + L.off_nd);
    float4 *ta = reinterpret_cast<float4 *>(smem + L.off_ta);
    float4 *tb = reinterpret_cast<float4 *>(smem + L.off_tb);
    float4 *tc = reinterpret_cast<float4 *>(smem + L.off_tc);
    for (int i = threadIdx.x; i < P.nodes_smem; i += blockDim.x) {
        sa[i] = P.node_a[i]; sb[i] = P.node_b[i]; sc[i] = P.node_c[i]; sd[i] = P.node_d[i];
    }
    for (int i = threadIdx.x; i < P.tris_smem; i += blockDim.x) {
        ta[i] = P.tri_a[i]; tb[i] = P.tri_b[i]; tc[i] = P.tri_c[i];
    }
    M.s_na = sa; M.s_nb = sb; M.s_nc = sc; M.s_nd = sd;
    M.s_ta = ta; M.s_tb = tb; M.s_tc = tc;
    M.nodes_smem = P.nodes_smem;
    M.tris_smem = P.tris_smem;
    M.n_nodes = P.n_nodes;
    M.n_tri = P.n_tri;
    M.dbg = P.counters ? P.counters + kBoundsCounter : nullptr;
    M.tri_eps = P.tri_eps;
    return M;
}

template <bool Exact, bool Grad, bool Agg = false>
__global__ void __launch_bounds__(kBlock, LP_TRANSPORT_MIN_BLOCKS) transport_kernel(const __grid_constant__ KParams P)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const SmemLayout L = smem_layout(P.nodes_smem, P.tris_smem);
    Medium *s_media = reinterpret_cast<Medium *>(smem + L.off_media);
    unsigned long long *s_region = reinterpret_cast<unsigned long long *>(smem + L.off_region);
    unsigned long long *s_cnt = reinterpret_cast<unsigned long long *>(smem + L.off_cnt);
    for (int i = threadIdx.x; i < P.n_media; i += blockDim.x) {
        s_media[i] = P.media[i];
        s_region[i] = 0;
    }
    if (threadIdx.x < 16) s_cnt[threadIdx.x] = 0;
    const MeshView M = stage_mesh(P, smem, L);
    __syncthreads();

    const unsigned lane = threadIdx.x & 31u;
    const unsigned lt_mask = (1u << lane) - 1u;
    Counters cnt = {};
    uint32_t photons = 0;
    Photon ph;
    GradAcc ga;
    bool alive = false;
    bool exhausted = false;
    for (;;) {
        const unsigned need = __ballot_sync(0xffffffffu, !alive);
        if (need && !exhausted) {
            const int k = __popc(need);
            unsigned long long base = 0;
            if (lane == 0) base = atomicAdd(P.work, (unsigned long long)k);
            base = __shfl_sync(0xffffffffu, base, 0);
            if (base + (unsigned long long)k >= (unsigned long long)P.n) exhausted = true;
            if (!alive) {
                const unsigned long long idx = base + __popc(need & lt_mask);
                if (idx < (unsigned long long)P.n) {
                    start_photon(P, ph, (uint32_t)idx);
                    if (Grad) {
                        for (int r = 0; r < P.n_media; ++r) {
                            ga.L[r] = 0.0f;
                            ga.k[r] = 0;
                        }
                    }
                    alive = true;
                }
            }
        }
        if (!__any_sync(0xffffffffu, alive)) break;
        if (alive) {
            if (!step_photon<Exact, Grad, kStackDepth, Agg>(P, M, s_media, s_region, s_cnt, ph, cnt, &ga)) {
                if (ph.region_acc) atomicAdd(s_region + ph.curr, ph.region_acc);
                if (Grad) {
                    ga.L[ph.curr] += ph.seg_len;
                    ga.k[ph.curr] += ph.seg_k;
                }
                finish_photon<Grad>(P, ph, Grad ? &ga : nullptr);
                photons++;
                alive = false;
            }
        }
    }
    // block-level reduction of counters and region sums
    const uint32_t cv[8] = {cnt.scatter, cnt.boundary, cnt.query, cnt.roulette, 0u, 0u, cnt.rz_drop, cnt.vox_drop};
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        if (i == 4 || i == 5) continue;
        unsigned long long x = cv[i];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0 && x) atomicAdd(s_cnt + i, x);
    }
    {
        unsigned long long x = photons;
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0 && x) atomicAdd(s_cnt + 8, x);
        x = cnt.skip;
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0 && x) atomicAdd(s_cnt + 10, x);
        x = cnt.bvh;
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0 && x) atomicAdd(s_cnt + 11, x);
    }
    __syncthreads();
    if (threadIdx.x < 16 && s_cnt[threadIdx.x]) atomicAdd(P.counters + threadIdx.x, s_cnt[threadIdx.x]);
    for (int i = threadIdx.x; i < P.n_media; i += blockDim.x)
        if (s_region[i]) atomicAdd(P.region + i, s_region[i]);
}

// P.grad selects the differentiating instantiation.
// The warp-aggregated form exists for the production arithmetic without differentiation
// only (P.agg_tallies is ignored otherwise).
template <bool Exact>
cudaError_t launch_transport_t(const KParams &P, int grid, int smem, cudaStream_t s)
{
    if (!Exact && !P.grad && P.agg_tallies) {
        cudaError_t e = cudaFuncSetAttribute(transport_kernel<false, false, true>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess) return e;
        transport_kernel<false, false, true><<<grid, kBlock, smem, s>>>(P);
    } else if (P.grad) {
        transport_kernel<Exact, true><<<grid, kBlock, smem, s>>>(P);
    } else {
        transport_kernel<Exact, false><<<grid, kBlock, smem, s>>>(P);
    }
    return cudaGetLastError();
}

template <bool Exact, bool Grad>
cudaError_t transport_occupancy_t(int smem, int *blocks_per_sm)
{
    cudaError_t e = cudaFuncSetAttribute(transport_kernel<Exact, Grad>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         smem);
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, transport_kernel<Exact, Grad>, kBlock, smem);
}

}  // namespace lp
