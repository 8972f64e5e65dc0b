/*
 * lp_oracle.c -- CPU oracle for the LightPropagation transport path.
 *
 * TEST INFRASTRUCTURE ONLY (see lp_oracle.h).  FP32 restatement of
 * src/Simulation/MCLightPropagation.cl and of the host binning in
 * src/Simulation/CalculatePropagation.cpp.  Build with -ffp-contract=off and
 * without fast-math: every expression below keeps the reference's evaluation
 * order so that the result is bit-identical to the reference kernel compiled for
 * the same CPU (pinned by tests/test_oracle_pin.py).
 */
#include "lp_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

/* ------------------------------------------------------------------ vectors */
typedef struct { float x, y, z; } f3;

static inline f3 mk(float x, float y, float z) { f3 r = {x, y, z}; return r; }
static inline f3 add(f3 a, f3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline f3 sub(f3 a, f3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline f3 scl(float s, f3 a) { return mk(s * a.x, s * a.y, s * a.z); }
static inline f3 neg(f3 a) { return mk(-a.x, -a.y, -a.z); }
/* OpenCL dot(): x*x + y*y + z*z evaluated left to right. */
static inline float dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline f3 cross(f3 a, f3 b)
{
    return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
/* OpenCL normalize(): v / |v|; a zero vector is returned unchanged. */
static inline f3 normalize(f3 v)
{
    float l = sqrtf(dot(v, v));
    if (l == 0.0f) return v;
    return mk(v.x / l, v.y / l, v.z / l);
}
/* OpenCL sign(). */
static inline float signf_cl(float x)
{
    if (x > 0.0f) return 1.0f;
    if (x < 0.0f) return -1.0f;
    if (x != x) return 0.0f;
    return x;
}
static inline f3 ld3(const float *a, int64_t i) { return mk(a[3 * i], a[3 * i + 1], a[3 * i + 2]); }

#define PI_F 3.14159265358979323846f

uint64_t lpo_fix(float w)
{
    /* w * 2^32 is exact in float; llrintf rounds to nearest even. */
    if (!(w > 0.0f)) return 0;
    return (uint64_t)llrintf(w * 4294967296.0f);
}

/* ------------------------------------------------------------------ Philox */
void lpo_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4])
{
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        c0 = hi1 ^ c1 ^ k0;
        c1 = lo1;
        c2 = hi0 ^ c3 ^ k1;
        c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* ------------------------------------------------------------------ ran3 */
void lpo_ran3_init(int32_t seed, float state56[56], int32_t inext3[3])
{
    /* PSNR::InitRand3 (PSNR.cpp:116-148) with ran3Seed = -|seed| (PSNR::SetSeed). */
    const long MBIG = 1000000000L, MSEED = 161803398L, MZ = 0;
    long ma[56];
    long idum = -labs((long)seed);
    long mj, mk;
    int i, ii, k, inext, inextp;
    memset(ma, 0, sizeof ma);
    mj = MSEED - (idum < 0 ? -idum : idum);
    mj %= MBIG;
    ma[55] = mj;
    mk = 1;
    for (i = 1; i <= 54; i++) {
        ii = (21 * i) % 55;
        ma[ii] = mk;
        mk = mj - mk;
        if (mk < MZ) mk += MBIG;
        mj = ma[ii];
    }
    for (k = 1; k <= 4; k++)
        for (i = 1; i <= 55; i++) {
            ma[i] -= ma[1 + (i + 30) % 55];
            if (ma[i] < MZ) ma[i] += MBIG;
        }
    inext = 0;
    inextp = 31;
    /* the first draw happens inside InitRand3 */
    if (++inext == 56) inext = 1;
    if (++inextp == 56) inextp = 1;
    mj = ma[inext] - ma[inextp];
    if (mj < MZ) mj += MBIG;
    ma[inext] = mj;
    for (i = 0; i < 56; i++) state56[i] = (float)ma[i]; /* GetRan3Array, PSNR.cpp:173-185 */
    inext3[0] = inext;
    inext3[1] = inextp;
    inext3[2] = 0;
}

float lpo_ran3_draw(float st[56], int32_t ix[3])
{
    /* DoRand3 (MCLightPropagation.cl:1204-1237): the table holds floats. */
    int a = ix[0] + 1, b = ix[1] + 1;
    if (a == 56) a = 1;
    if (b == 56) b = 1;
    float r = st[a] - st[b];
    if (r < 0) r += (float)1000000000L;
    st[a] = r;
    ix[0] = a;
    ix[1] = b;
    ix[2] = 0;
    return r / (float)1000000000L;
}

/* ------------------------------------------------------------------ RNG */
typedef struct {
    int mode;
    /* ran3 */
    float *st;
    int32_t *ix;
    float own_st[56];
    int32_t own_ix[3];
    /* philox */
    uint32_t key[2], ctr[4], buf[4];
    uint64_t draws;
} rng_t;

/* Draw slots of one transport event (shared with the CUDA path). */
enum { SLOT_STEP = 0, SLOT_ANGLE = 1, SLOT_AZIMUTH = 2, SLOT_ROULETTE = 3 };

static void rng_photon(rng_t *r, const lpo_problem *P, int64_t pid)
{
    r->draws = 0;
    if (r->mode == LPO_RNG_RAN3_PHOTON) {
        int32_t s = (int32_t)(1 + (int64_t)(((uint64_t)P->seed * 1000003ull + (uint64_t)pid) % 161803397ull));
        lpo_ran3_init(s, r->own_st, r->own_ix);
        r->st = r->own_st;
        r->ix = r->own_ix;
    } else if (r->mode == LPO_RNG_PHILOX) {
        r->key[0] = (uint32_t)P->seed;
        r->key[1] = (uint32_t)(P->seed >> 32);
        r->ctr[0] = (uint32_t)(uint64_t)pid;
        r->ctr[1] = (uint32_t)((uint64_t)pid >> 32);
        r->ctr[2] = 0;
        r->ctr[3] = P->stream;
    }
}

/* Philox layout shared with the CUDA path: one Philox4x32-10 block per event,
 * counter = (photon lo, photon hi, event, stream), key = seed.  Event 0 samples the
 * source; transport loop iteration i (0-based) is event i + 1.  The block's four
 * words are the event's draw slots (step, Fresnel or polar angle, azimuth,
 * roulette), each mapped to the odd multiple of 2^-24 ((x >> 8) | 1) * 2^-24, a
 * uniform in (0, 1).  The ran3 modes ignore events and slots and draw in order,
 * which is the reference's draw order within an event. */
static inline void rng_event(rng_t *r, uint32_t ev)
{
    if (r->mode == LPO_RNG_PHILOX) {
        r->ctr[2] = ev;
        lpo_philox4x32_10(r->ctr, r->key, r->buf);
    }
}

static inline float rng_slot(rng_t *r, int slot)
{
    r->draws++;
    if (r->mode == LPO_RNG_PHILOX) return (float)((r->buf[slot] >> 8) | 1u) * 0x1.0p-24f;
    return lpo_ran3_draw(r->st, r->ix);
}

/* ------------------------------------------------------------------ geometry */
void lpo_geometry_of(const float dimensions[3], const float det_grid[6], lpo_geometry *g)
{
    /* CalculatePropagation::InitLogVectors (CP.cpp:120-131): float divisions, int casts. */
    g->dimx = (int32_t)(dimensions[0] / det_grid[0]);
    g->dimy = (int32_t)(dimensions[1] / det_grid[1]);
    g->dimz = (int32_t)(dimensions[2] / det_grid[2]);
    g->dimAlpha = (int32_t)(90 / det_grid[5]);
    g->dimR = (int32_t)ceil(sqrt(pow((double)(g->dimx / 2), 2) + pow((double)(g->dimy / 2), 2)));
    g->sft_nx = 2 * (g->dimx / 2) + 1;
    g->sft_ny = 2 * (g->dimy / 2) + 1;
    g->rz_nr = 2 * g->dimR + 1;
    g->rz_nz = g->dimz + 1;
    /* The kernel recomputes dimR from the float dims (MCLightPropagation.cl:263). */
    float hx = (float)g->dimx / 2, hy = (float)g->dimy / 2;
    g->kernel_dimR = (int32_t)ceilf(sqrtf(powf(hx, 2.0f) + powf(hy, 2.0f)));
}

float lpo_rspecular(const float *nm)
{
    /* Rspecular (MCLightPropagation.cl:273-299). */
    float r1, r2, temp;
    float n1 = nm[0];
    float n2 = nm[4], mua1 = nm[5], mus1 = nm[6];
    temp = (n1 - n2) / (n1 + n2);
    r1 = temp * temp;
    if (mua1 == 0.0f && mus1 == 0.0f) {
        float n3 = nm[8];
        temp = (n2 - n3) / (n2 + n3);
        r2 = temp * temp;
        r1 = r1 + (1 - r1) * (1 - r1) * r2 / (1 - r1 * r2);
    }
    return r1;
}

float lpo_fresnel(float n1, float n2, float cosIn)
{
    /* GetFresnel (MCLightPropagation.cl:857-907). */
    float r;
    if (n1 == n2) {
        r = 0.0f;
    } else if (fabsf(cosIn) == 1.0f) {
        r = (n1 - n2) / (n1 + n2);
        r *= r;
    } else if (cosIn == 0.0f) {
        r = 1.0f;
    } else {
        float sinIn = sqrtf(1 - cosIn * cosIn);
        float sinOut = n1 * sinIn / n2;
        if (sinOut >= 1.0f) {
            r = 1.0f;
        } else {
            float cosOut = sqrtf(1 - sinOut * sinOut);
            float cap = cosIn * cosOut - sinIn * sinOut;
            float cam = cosIn * cosOut + sinIn * sinOut;
            float sap = sinIn * cosOut + cosIn * sinOut;
            float sam = sinIn * cosOut - cosIn * sinOut;
            r = 0.5f * (sam * sam) * ((cam * cam) + (cap * cap)) / ((sap * sap) * (cam * cam));
        }
    }
    return r;
}

float lpo_hg_cos_theta(float g, float xi)
{
    /* VScatter (MCLightPropagation.cl:625-634). */
    float cosTheta = 0;
    float g1 = (1 - g * g) / (1 - g + 2 * g * xi);
    if (g != 0) {
        cosTheta = (1 + g * g - g1 * g1) / (2 * g);
        if (cosTheta < -1) cosTheta = -1;
        else if (cosTheta > 1) cosTheta = 1;
    } else {
        cosTheta = 2 * xi - 1;
    }
    return cosTheta;
}

int32_t lpo_find_triangle(const float *tri, int32_t n_tri, int32_t ref_tri,
                          const float pp[3], const float vv[3], float *t_out)
{
    /* PhotonClass::FindTriangleInPath (MCLightPropagation.cl:1037-1093). */
    f3 p = mk(pp[0], pp[1], pp[2]), v = mk(vv[0], vv[1], vv[2]);
    float best = 10000;
    int32_t id = -1;
    for (int32_t j = 0; j < n_tri; j++) {
        if (j == ref_tri) continue;
        f3 K = ld3(tri, 3 * (int64_t)j), L = ld3(tri, 3 * (int64_t)j + 1), M = ld3(tri, 3 * (int64_t)j + 2);
        f3 E = sub(K, M), F = sub(L, M), G = sub(p, M);
        float t = dot(cross(G, E), F);
        float w = dot(cross(v, F), E);
        float k = dot(cross(v, F), G);
        float l = dot(cross(G, E), v);
        t /= w;
        k /= w;
        l /= w;
        if (t < best && t > 0.0f && k >= 0.0f && l >= 0.0f && (k + l) < 1) {
            best = t;
            id = j;
        }
    }
    *t_out = best;
    return id;
}

/* ------------------------------------------------------------------ photon */
typedef struct {
    f3 v, p, SFT;
    float w, stepsize, steptoboundary, unfin, absorbed;
    int fetal, refTri;
} photon_t;

/* Rotate (MCLightPropagation.cl:697-708). */
static inline f3 rotate(f3 vec, f3 axis, float c, float s)
{
    float nDx = dot(axis, vec);
    f3 nXx = cross(axis, vec);
    f3 nXxXn = cross(nXx, axis);
    return add(add(scl(nDx, axis), scl(c, nXxXn)), scl(s, nXx));
}

/* VScatter (MCLightPropagation.cl:597-655). */
static void vscatter(photon_t *ph, float g, float xt, float xp)
{
    f3 v = ph->v;
    f3 e_rot = mk(0, 0, 0);
    if (v.z != 0.0f) {
        float z = -(v.x + v.y) / (v.z);
        e_rot = mk(1, 1, z);
    } else if (v.y != 0.0f) {
        float y = -(v.x) / (v.y);
        e_rot = mk(1, y, 0);
    } else if (v.x != 0.0f) {
        e_rot = mk(0, 1, 0);
    }
    e_rot = normalize(e_rot);
    float cosTheta = lpo_hg_cos_theta(g, xt);
    float sinTheta = sqrtf(1.0f - cosTheta * cosTheta);
    float psi = 2 * PI_F * xp;
    float cosPsi = cosf(psi);
    float sinPsi = sqrtf(1.0f - cosPsi * cosPsi);
    if (psi > PI_F) sinPsi *= -1;
    f3 rot_theta = normalize(rotate(v, e_rot, cosTheta, sinTheta));
    ph->v = normalize(rotate(rot_theta, v, cosPsi, sinPsi));
}

/* Transmit / Reflect (MCLightPropagation.cl:506-549). */
static void transmit(photon_t *ph, f3 e_x, float d, float n1, float n2)
{
    f3 e_y = normalize(cross(e_x, cross(e_x, ph->v)));
    float sinT = sqrtf(1 - d * d) * n1 / n2;
    float cosT = -sqrtf(1 - sinT * sinT);
    if (d > 0.0f) cosT = fabsf(cosT);
    ph->v = normalize(sub(scl(cosT, e_x), scl(sinT, e_y)));
}
static void reflect(photon_t *ph, f3 e_x, float d)
{
    f3 e_y = normalize(cross(e_x, cross(e_x, ph->v)));
    float sinR = sqrtf(1 - d * d);
    ph->v = neg(normalize(add(scl(d, e_x), scl(sinR, e_y))));
}

typedef struct {
    const lpo_problem *P;
    lpo_geometry g;
    f3 eX, eY, eZ, POI, nX, nY, nZ;
    float Rsp, distMin, exitScale;
} ctx_t;

/* TransmitOrReflect (MCLightPropagation.cl:921-1018). */
static int transmit_or_reflect(const ctx_t *C, photon_t *ph, const float *cur, const float *nxt,
                               f3 nv, int curr, int inner, int outer, float xi)
{
    int newID;
    float muaNew, musNew;
    float cosIn = dot(nv, ph->v);
    float absCosIn = fabsf(cosIn);
    float n1 = cur[0], n2 = nxt[0];
    float cos_crit = 0.0f;
    if (n1 > n2) cos_crit = sqrtf(1.0f - (n2 / n1) * (n2 / n1));
    float r;
    if (absCosIn <= cos_crit) r = 1.0f;
    else r = lpo_fresnel(n1, n2, (C->P->compat & LPO_COMPAT_SIGNED_FRESNEL) ? cosIn : absCosIn);
    if (xi > r) {
        transmit(ph, nv, cosIn, n1, n2);
        newID = (cosIn > 0) ? outer : inner;
        muaNew = nxt[1];
        musNew = nxt[2];
    } else {
        reflect(ph, nv, cosIn);
        newID = curr;
        muaNew = cur[1];
        musNew = cur[2];
    }
    if (muaNew == 0 || musNew == 0) {
        float scale = (C->P->compat & LPO_COMPAT_EXIT_RSP) ? (1 - C->Rsp) : 1.0f;
        ph->SFT.y = 0;
        float dist = fabsf(dot(C->nZ, sub(ph->p, C->POI)));
        if (dist > C->distMin) {
            ph->SFT.z = ph->w * scale;
        } else {
            if (ph->fetal) ph->SFT.y = ph->w * scale;
            ph->SFT.x = ph->w * scale;
        }
        ph->w = 0;
    }
    return newID;
}

static inline void tally_add(uint64_t *a, float w) { *a += lpo_fix(w); }

/* One absorption deposit: r-z grid, voxel grid, reference-layout r-z buffer. */
static void record_absorption(const ctx_t *C, lpo_tallies *T, f3 coords, float dw, float mua,
                              const float *det_grid)
{
    const lpo_problem *P = C->P;
    /* RecordAbsorbtionRZ (MCLightPropagation.cl:254-271): signed radius in dr units */
    float radius = sqrtf(coords.x * coords.x + coords.y * coords.y) * signf_cl(coords.x) / det_grid[3];
    if (T->rz_ref) {
        int kR = C->g.kernel_dimR;
        int id = (int)(coords.z * (2 * kR + 1) / det_grid[2] + radius + kR);
        int64_t cell = (int64_t)id + T->rz_ref_offset;
        if (cell >= 0 && cell < T->rz_ref_cells) {
            float *c = T->rz_ref + 3 * cell;
            c[0] = 1;
            c[1] = c[1] + dw;
            c[2] = mua;
        } else {
            T->counters[LPO_C_RZ_DROP] += 1000000; /* flags an out-of-buffer reference index */
        }
    }
    if (T->rz) {
        int row = (int)floorf(coords.z / det_grid[2]);
        int col = (int)floorf(radius + (float)C->g.dimR);
        if (row >= 0 && row < C->g.rz_nz && col >= 0 && col < C->g.rz_nr) {
            uint64_t *c = T->rz + 2 * ((int64_t)row * C->g.rz_nr + col);
            tally_add(&c[0], dw);
            if (mua > 0) tally_add(&c[1], dw / mua);
        } else {
            T->counters[LPO_C_RZ_DROP]++;
        }
    }
    if (T->vox && P->vox_n[0] > 0) {
        int ix = (int)floorf(coords.x / P->vox_d[0] + 0.5f * (float)P->vox_n[0]);
        int iy = (int)floorf(coords.y / P->vox_d[1] + 0.5f * (float)P->vox_n[1]);
        int iz = (int)floorf(coords.z / P->vox_d[2]);
        if (ix >= 0 && ix < P->vox_n[0] && iy >= 0 && iy < P->vox_n[1] && iz >= 0 && iz < P->vox_n[2])
            tally_add(&T->vox[((int64_t)iz * P->vox_n[1] + iy) * P->vox_n[0] + ix], dw);
        else
            T->counters[LPO_C_VOX_DROP]++;
    }
}

static inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

/* float -> int truncation that maps NaN to 0 and saturates far outside the grid. */
static inline int trunc_sat(double x)
{
    if (x != x) return 0;
    if (x > 1e9) return 1000000000;
    if (x < -1e9) return -1000000000;
    return (int)x;
}

/* Host binning of one exit record (CalculatePropagation.cpp:1553-1626). */
static void bin_exit(const ctx_t *C, lpo_tallies *T, const float rec[8], const double *L, const int64_t *K)
{
    const lpo_problem *P = C->P;
    const lpo_geometry *g = &C->g;
    const float *dg = P->det_grid;
    float s = rec[3], f = rec[4], t = rec[5];
    if (s == 0.0f && f == 0.0f && t == 0.0f) return;
    int hx = g->dimx / 2, hy = g->dimy / 2;
    int x = trunc_sat(rec[0] / dg[0]);
    int y = trunc_sat(rec[1] / dg[1]);
    y = clampi(y, -hy, hy);
    x = clampi(x, -hx, hx);
    uint64_t *c = T->sft + 3 * ((int64_t)(y + hy) * g->sft_nx + (x + hx));
    tally_add(&c[0], s);
    tally_add(&c[1], f);
    tally_add(&c[2], t);
    int ai = trunc_sat(((double)(rec[6] * 180) / 3.14159265358979323846) / (double)dg[5]);
    int ri = trunc_sat(rec[7] / dg[3]);
    if (ri > g->dimR - 1) ri = g->dimR - 1;
    else if (ri < 0) ri = 0;
    if (ai > g->dimAlpha - 1) ai = g->dimAlpha - 1;
    else if (ai < 0) ai = 0;
    uint64_t *r = T->rtd + 3 * ((int64_t)ai * g->dimR + ri);
    tally_add(&r[0], s);
    tally_add(&r[1], f);
    tally_add(&r[2], t);
    /* radial exit bins and ring detectors: radius in the emitter plane */
    float rho = sqrtf(rec[0] * rec[0] + rec[1] * rec[1]);
    if (T->rbins && P->n_rbins > 0) {
        int b = trunc_sat(rho / P->rbin_dr);
        if (b >= 0 && b < P->n_rbins) {
            tally_add(&T->rbins[2 * b], s);
            tally_add(&T->rbins[2 * b + 1], t);
        }
    }
    if (T->det && s > 0.0f) {
        for (int d = 0; d < P->n_det; d++) {
            if (rho >= P->det_r[2 * d] && rho < P->det_r[2 * d + 1]) {
                tally_add(&T->det[2 * d], s);
                tally_add(&T->det[2 * d + 1], s * s);
                if (T->grad && L) {
                    for (int r = 0; r < P->n_media; r++) {
                        double a = (double)s * L[r], b = (double)s * (double)K[r];
                        double *g = T->grad + 5 * ((int64_t)d * P->n_media + r);
                        g[0] += a;
                        g[1] += b;
                        g[2] += a * a;
                        g[3] += b * b;
                        g[4] += a * b;
                    }
                }
            }
        }
    }
}

/* The kernel body for one photon (MCLightPropagation.cl:1287-1597). */
static void trace_photon(const ctx_t *C, rng_t *R, int64_t pid, lpo_tallies *T, float *rec_out)
{
    const lpo_problem *P = C->P;
    const float *nm = P->nmuasg;
    const float *dg = P->det_grid;
    photon_t ph;
    rng_photon(R, P, pid);
    /* PhotonClass::Init (.cl:344-389) with vStart[0] (.cl:429-467) */
    ph.v = mk(P->v_start[0], P->v_start[1], P->v_start[2]);
    ph.p = mk(P->p_start[0], P->p_start[1], P->p_start[2]);
    if (P->src_type == 1) {
        /* fibre source (extension, see lp_oracle.h), event 0 */
        rng_event(R, 0);
        float x1 = rng_slot(R, 0), x2 = rng_slot(R, 1), x3 = rng_slot(R, 2), x4 = rng_slot(R, 3);
        float r = P->src_radius * sqrtf(x1);
        float phi = 2 * PI_F * x2;
        float cp = cosf(phi), sp = sinf(phi);
        ph.p = add(ph.p, add(scl(r * cp, C->nX), scl(r * sp, C->nY)));
        float ct = 1.0f - x3 * (1.0f - P->src_cos_max);
        float stt = sqrtf(1.0f - ct * ct);
        float psi = 2 * PI_F * x4;
        float cq = cosf(psi), sq = sinf(psi);
        ph.v = normalize(add(scl(ct, C->nZ), add(scl(stt * cq, C->nX), scl(stt * sq, C->nY))));
    }
    ph.w = 1.0f - C->Rsp;
    ph.SFT = mk(0, 0, 0);
    ph.stepsize = 0.0f;
    ph.unfin = 0.0f;
    ph.fetal = 0;
    ph.refTri = -1;
    ph.absorbed = 0.0f;
    ph.steptoboundary = 0.0f;
    int curr = 0;
    f3 nv = mk(0, 0, -1);
    int roulette = 1;
    int64_t steps = 0;
    uint64_t region_acc = 0;
    /* path length and interactions per region, for the perturbation-MC sums */
    double L[LPO_MAX_MEDIA];
    int64_t K[LPO_MAX_MEDIA];
    const int track = T->grad != NULL && P->n_media <= LPO_MAX_MEDIA;
    if (track) {
        memset(L, 0, sizeof L);
        memset(K, 0, sizeof K);
    }
    do {
        float pp[3] = {ph.p.x, ph.p.y, ph.p.z}, vv[3] = {ph.v.x, ph.v.y, ph.v.z};
        int triID = lpo_find_triangle(P->tri, P->n_tri, ph.refTri, pp, vv, &ph.steptoboundary);
        T->counters[LPO_C_QUERY]++;
        rng_event(R, (uint32_t)(steps + 1));
        const float *cur = nm + 4 * curr;
        if (cur[1] == 0.0f && cur[2] == 0.0f) {
            ph.stepsize = ph.steptoboundary;
        } else if (ph.unfin == 0.0f) {
            float xi;
            do { xi = rng_slot(R, SLOT_STEP); } while (xi <= 0.0f);
            ph.stepsize = -logf(xi) * P->factor / (cur[1] + cur[2]);
        } else {
            ph.stepsize = ph.unfin / (cur[1] + cur[2]);
            ph.unfin = 0.0f;
        }
        if (ph.steptoboundary <= ph.stepsize) {
            T->counters[LPO_C_BOUNDARY]++;
            ph.p = add(ph.p, scl(ph.steptoboundary, ph.v));
            ph.refTri = -1;
            float xi = rng_slot(R, SLOT_ANGLE);
            if (triID < 0) {
                /* no triangle ahead: the reference reads mediumIDs[-1]; here the photon leaves */
                T->counters[LPO_C_MISS]++;
                ph.w = 0;
            } else {
                if (track) L[curr] += ph.steptoboundary;
                int inner = P->med[2 * triID], outer = P->med[2 * triID + 1];
                if (curr != inner && curr != outer) T->counters[LPO_C_MISMATCH]++;
                nv = normalize(ld3(P->nrm, triID));
                const float *nxt = (curr == outer) ? nm + 4 * inner : nm + 4 * outer;
                if (P->compat & LPO_COMPAT_AXIS_NORMAL) {
                    f3 cs = ph.p;
                    if (fabsf(sqrtf(cs.x * cs.x + cs.y * cs.y)) < 0.01f)
                        nv = scl(signf_cl(dot(nv, C->eZ)), C->nZ);
                }
                int prev = curr;
                curr = transmit_or_reflect(C, &ph, cur, nxt, nv, curr, inner, outer, xi);
                ph.refTri = triID;
                if (curr == P->fetal_id) ph.fetal = 1;
                ph.unfin = (ph.stepsize - ph.steptoboundary) * (cur[1] + cur[2]);
                if (curr != prev && T->region) {
                    T->region[prev] += region_acc;
                    region_acc = 0;
                }
            }
        } else {
            T->counters[LPO_C_SCATTER]++;
            ph.p = add(ph.p, scl(ph.stepsize, ph.v));
            ph.refTri = -1;
            if (track) {
                L[curr] += ph.stepsize;
                K[curr]++;
            }
            /* Absorb (.cl:841-847) */
            if (cur[1] > 0.0f && cur[2] > 0.0f) {
                ph.absorbed = ph.w * (cur[1] / (cur[1] + cur[2]));
                ph.w -= ph.absorbed;
            }
            float xt = rng_slot(R, SLOT_ANGLE);
            float xp = rng_slot(R, SLOT_AZIMUTH);
            vscatter(&ph, cur[3], xt, xp);
            f3 pr = sub(ph.p, C->POI);
            f3 coords = mk(dot(C->nX, pr), dot(C->nY, pr), dot(C->nZ, pr));
            record_absorption(C, T, coords, ph.absorbed, cur[1], dg);
            region_acc += lpo_fix(ph.absorbed);
        }
        if (ph.w < P->w_threshold && ph.w > 0.0f) {
            float xi = rng_slot(R, SLOT_ROULETTE);
            T->counters[LPO_C_ROULETTE]++;
            if (xi < P->chance) {
                ph.w /= P->chance;
                roulette = 1;
            } else {
                ph.w = 0;
                roulette = 0;
            }
        }
        steps++;
        if (P->max_steps > 0 && steps >= P->max_steps && ph.w > 0.0f) {
            T->counters[LPO_C_CAPPED]++;
            ph.w = 0;
        }
    } while (ph.w > 0.0f && (ph.w > P->w_threshold || roulette));
    if (T->region) T->region[curr] += region_acc;
    T->counters[LPO_C_PHOTONS]++;
    T->counters[LPO_C_DRAWS] += R->draws;
    /* exit record (.cl:1583-1594) */
    float rec[8];
    float alpha = fabsf(acosf(dot(ph.v, nv)));
    f3 d = sub(C->POI, ph.p);
    float radius = sqrtf(d.x * d.x + d.y * d.y + d.z * d.z);
    f3 pr = sub(ph.p, C->POI);
    rec[0] = dot(C->nX, pr);
    rec[1] = dot(C->nY, pr);
    rec[2] = dot(C->nZ, pr);
    rec[3] = ph.SFT.x;
    rec[4] = ph.SFT.y;
    rec[5] = ph.SFT.z;
    rec[6] = alpha;
    rec[7] = radius;
    if (rec_out) memcpy(rec_out, rec, sizeof rec);
    bin_exit(C, T, rec, track ? L : NULL, track ? K : NULL);
}

static void ctx_init(ctx_t *C, const lpo_problem *P)
{
    C->P = P;
    lpo_geometry_of(P->dimensions, P->det_grid, &C->g);
    C->POI = mk(P->ep0xyz[0], P->ep0xyz[1], P->ep0xyz[2]);
    C->eX = mk(P->ep0xyz[3], P->ep0xyz[4], P->ep0xyz[5]);
    C->eY = mk(P->ep0xyz[6], P->ep0xyz[7], P->ep0xyz[8]);
    C->eZ = mk(P->ep0xyz[9], P->ep0xyz[10], P->ep0xyz[11]);
    C->nX = normalize(C->eX);
    C->nY = normalize(C->eY);
    C->nZ = normalize(C->eZ);
    C->Rsp = lpo_rspecular(P->nmuasg);
    /* distMin = gridDimsXYZ.z * dimsXYZ[2] / 2 (.cl:1351) */
    C->distMin = P->det_grid[2] * (float)C->g.dimz / 2.0f;
}

/* ------------------------------------------------------------------ driver */
typedef struct {
    ctx_t *C;
    int64_t first, n, chunk;
    int64_t *next;
    pthread_mutex_t *lock;
    lpo_tallies T;
    lpo_tallies *out;
} worker_t;

static size_t n_sft(const lpo_geometry *g) { return (size_t)g->sft_nx * g->sft_ny * 3; }
static size_t n_rtd(const lpo_geometry *g) { return (size_t)g->dimR * g->dimAlpha * 3; }
static size_t n_rz(const lpo_geometry *g) { return (size_t)g->rz_nr * g->rz_nz * 2; }
static size_t n_vox(const lpo_problem *P)
{
    return P->vox_n[0] > 0 ? (size_t)P->vox_n[0] * P->vox_n[1] * P->vox_n[2] : 0;
}

static void *worker_main(void *arg)
{
    worker_t *W = (worker_t *)arg;
    rng_t R;
    memset(&R, 0, sizeof R);
    R.mode = W->C->P->rng_mode;
    for (;;) {
        int64_t s;
        pthread_mutex_lock(W->lock);
        s = *W->next;
        *W->next += W->chunk;
        pthread_mutex_unlock(W->lock);
        if (s >= W->n) break;
        int64_t e = s + W->chunk < W->n ? s + W->chunk : W->n;
        for (int64_t i = s; i < e; i++)
            trace_photon(W->C, &R, W->first + i, &W->T,
                         W->out->exit_rec ? W->out->exit_rec + 8 * i : NULL);
    }
    return NULL;
}

static void merge(uint64_t *dst, const uint64_t *src, size_t n)
{
    if (!dst || !src) return;
    for (size_t i = 0; i < n; i++) dst[i] += src[i];
}

int lpo_run(const lpo_problem *P, int64_t first, int64_t n, int nthreads,
            float *ran3_state, int32_t *ran3_inext, lpo_tallies *T)
{
    ctx_t C;
    ctx_init(&C, P);
    if (n <= 0) return 0;
    if (P->rng_mode == LPO_RNG_RAN3_SHARED) {
        rng_t R;
        memset(&R, 0, sizeof R);
        R.mode = LPO_RNG_RAN3_SHARED;
        R.st = ran3_state;
        R.ix = ran3_inext;
        for (int64_t i = 0; i < n; i++)
            trace_photon(&C, &R, first + i, T, T->exit_rec ? T->exit_rec + 8 * i : NULL);
        return 0;
    }
    if (nthreads <= 0) nthreads = (int)sysconf(_SC_NPROCESSORS_ONLN);
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    int64_t next = 0;
    pthread_mutex_t lock = PTHREAD_MUTEX_INITIALIZER;
    worker_t *W = (worker_t *)calloc((size_t)nthreads, sizeof(worker_t));
    pthread_t *th = (pthread_t *)calloc((size_t)nthreads, sizeof(pthread_t));
    int64_t chunk = n / ((int64_t)nthreads * 16);
    if (chunk < 1) chunk = 1;
    if (chunk > 4096) chunk = 4096;
    for (int t = 0; t < nthreads; t++) {
        worker_t *w = &W[t];
        w->C = &C;
        w->first = first;
        w->n = n;
        w->chunk = chunk;
        w->next = &next;
        w->lock = &lock;
        w->out = T;
        w->T.sft = T->sft ? (uint64_t *)calloc(n_sft(&C.g), 8) : NULL;
        w->T.rtd = T->rtd ? (uint64_t *)calloc(n_rtd(&C.g), 8) : NULL;
        w->T.rz = T->rz ? (uint64_t *)calloc(n_rz(&C.g), 8) : NULL;
        w->T.vox = (T->vox && n_vox(P)) ? (uint64_t *)calloc(n_vox(P), 8) : NULL;
        w->T.rbins = (T->rbins && P->n_rbins > 0) ? (uint64_t *)calloc((size_t)P->n_rbins * 2, 8) : NULL;
        w->T.region = T->region ? (uint64_t *)calloc((size_t)P->n_media, 8) : NULL;
        w->T.det = (T->det && P->n_det > 0) ? (uint64_t *)calloc((size_t)P->n_det * 2, 8) : NULL;
        w->T.grad = (T->grad && P->n_det > 0) ? (double *)calloc((size_t)P->n_det * P->n_media * 5, 8) : NULL;
        w->T.exit_rec = NULL;
        w->T.rz_ref = NULL; /* the reference-layout buffer is only kept in the sequential mode */
        if (t > 0) pthread_create(&th[t], NULL, worker_main, w);
    }
    worker_main(&W[0]);
    for (int t = 1; t < nthreads; t++) pthread_join(th[t], NULL);
    for (int t = 0; t < nthreads; t++) {
        worker_t *w = &W[t];
        merge(T->sft, w->T.sft, n_sft(&C.g));
        merge(T->rtd, w->T.rtd, n_rtd(&C.g));
        merge(T->rz, w->T.rz, n_rz(&C.g));
        merge(T->vox, w->T.vox, n_vox(P));
        merge(T->rbins, w->T.rbins, (size_t)P->n_rbins * 2);
        merge(T->region, w->T.region, (size_t)P->n_media);
        merge(T->det, w->T.det, (size_t)P->n_det * 2);
        if (T->grad && w->T.grad)
            for (size_t k = 0; k < (size_t)P->n_det * P->n_media * 5; k++) T->grad[k] += w->T.grad[k];
        for (int k = 0; k < LPO_NCOUNTERS; k++) T->counters[k] += w->T.counters[k];
        free(w->T.sft); free(w->T.rtd); free(w->T.rz); free(w->T.vox);
        free(w->T.rbins); free(w->T.region); free(w->T.det); free(w->T.grad);
    }
    free(W);
    free(th);
    return 0;
}
