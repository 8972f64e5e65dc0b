/*
 * lp_oracle64.c -- FP64 error oracle for the LightPropagation transport path.
 *
 * TEST INFRASTRUCTURE ONLY (see lp_oracle.h): the checker for the stated error of the
 * CUDA path, never the product.  It traces the same physics as the FP32 restatement in
 * lp_oracle.c -- the reference kernel src/Simulation/MCLightPropagation.cl:1262-1606
 * and the host binning of src/Simulation/CalculatePropagation.cpp:1553-1626 -- with
 * every quantity (position, direction, weight, step, Fresnel, scattering angles,
 * tally coordinates) in double precision:
 *   - step length        .cl:1405-1442   (-ln xi * factor / (mua + mus), or residual)
 *   - nearest triangle   .cl:1037-1093   (same intersection formulas, in double; the
 *                                         search runs over a bounding-volume tree of
 *                                         the mesh, lpo64_mesh, and returns the
 *                                         brute-force scan's answer: nearest t, then
 *                                         lowest triangle index)
 *   - boundary           .cl:857-1018    (GetFresnel, critical angle, Transmit/Reflect,
 *                                         exit scoring)
 *   - absorb / scatter   .cl:841-854, 597-655, 697-708 (VScatter with Rodrigues rotations)
 *   - roulette           .cl:1020-1035
 *   - tallies            .cl:101-115, 254-271 and CP.cpp:1553-1626, in the fixed-point
 *                        layouts of lpo_tallies
 * Random numbers: the Philox counter layout of the CUDA path and of lp_oracle.c (one
 * block per event, four draw slots), each slot mapped to the same 24-bit uniform.  A
 * photon therefore consumes the same random numbers as in the FP32 oracle and on the
 * GPU, and follows the same trajectory until a rounding difference flips a decision.
 * The reference quirks Q3, Q4 and Q10 follow the compat bits exactly as in lp_oracle.c.
 */
#include "lp_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

typedef struct { double x, y, z; } d3;

static inline d3 mk(double x, double y, double z) { d3 r = {x, y, z}; return r; }
static inline d3 add(d3 a, d3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline d3 sub(d3 a, d3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline d3 scl(double s, d3 a) { return mk(s * a.x, s * a.y, s * a.z); }
static inline d3 neg(d3 a) { return mk(-a.x, -a.y, -a.z); }
static inline double dot(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline d3 cross(d3 a, d3 b)
{
    return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline d3 normalize(d3 v)
{
    double l = sqrt(dot(v, v));
    if (l == 0.0) return v;
    return mk(v.x / l, v.y / l, v.z / l);
}
static inline double sign_cl(double x)
{
    if (x > 0.0) return 1.0;
    if (x < 0.0) return -1.0;
    return x;
}
static inline d3 ldf3(const float *a, int64_t i)
{
    return mk((double)a[3 * i], (double)a[3 * i + 1], (double)a[3 * i + 2]);
}

#define PI_D 3.14159265358979323846
#define NOHIT 10000.0

static inline uint64_t fix64(double w)
{
    if (!(w > 0.0)) return 0;
    return (uint64_t)llrint(w * 4294967296.0);
}

/* ------------------------------------------------------------------ mesh + tree */
/* Triangle records in double: M, E = K - M, F = L - M (the reference's operands). */
typedef struct { double m[3], e[3], f[3]; int32_t id; } tri64;
typedef struct { double lo[3], hi[3]; int32_t left, right, first, count; } node64;

struct lpo64_mesh {
    int32_t n_tri, n_nodes;
    tri64 *tris;     /* in tree order */
    node64 *nodes;
};

typedef struct { double lo[3], hi[3], c[3]; int32_t id; } prim_t;

static int cmp_axis;
static int prim_cmp(const void *a, const void *b)
{
    double x = ((const prim_t *)a)->c[cmp_axis], y = ((const prim_t *)b)->c[cmp_axis];
    if (x < y) return -1;
    if (x > y) return 1;
    return ((const prim_t *)a)->id - ((const prim_t *)b)->id;
}

/* Median split on the longest centroid axis, leaves of at most 4 triangles. */
static int32_t build_node(struct lpo64_mesh *M, prim_t *p, int32_t first, int32_t count, int32_t *n_nodes)
{
    int32_t me = (*n_nodes)++;
    node64 *nd = &M->nodes[me];
    double clo[3] = {1e300, 1e300, 1e300}, chi[3] = {-1e300, -1e300, -1e300};
    for (int k = 0; k < 3; k++) { nd->lo[k] = 1e300; nd->hi[k] = -1e300; }
    for (int32_t i = first; i < first + count; i++)
        for (int k = 0; k < 3; k++) {
            if (p[i].lo[k] < nd->lo[k]) nd->lo[k] = p[i].lo[k];
            if (p[i].hi[k] > nd->hi[k]) nd->hi[k] = p[i].hi[k];
            if (p[i].c[k] < clo[k]) clo[k] = p[i].c[k];
            if (p[i].c[k] > chi[k]) chi[k] = p[i].c[k];
        }
    if (count <= 4) {
        nd->left = nd->right = -1;
        nd->first = first;
        nd->count = count;
        return me;
    }
    int axis = 0;
    for (int k = 1; k < 3; k++)
        if (chi[k] - clo[k] > chi[axis] - clo[axis]) axis = k;
    cmp_axis = axis;
    qsort(p + first, (size_t)count, sizeof(prim_t), prim_cmp);
    int32_t half = count / 2;
    nd->first = first;
    nd->count = 0;
    int32_t l = build_node(M, p, first, half, n_nodes);
    int32_t r = build_node(M, p, first + half, count - half, n_nodes);
    M->nodes[me].left = l;
    M->nodes[me].right = r;
    return me;
}

lpo64_mesh *lpo64_mesh_build(const float *tri, int32_t n_tri)
{
    struct lpo64_mesh *M = (struct lpo64_mesh *)calloc(1, sizeof *M);
    M->n_tri = n_tri;
    if (n_tri <= 0) return M;
    prim_t *p = (prim_t *)malloc(sizeof(prim_t) * (size_t)n_tri);
    for (int32_t j = 0; j < n_tri; j++) {
        for (int k = 0; k < 3; k++) {
            double a = tri[9 * (int64_t)j + k], b = tri[9 * (int64_t)j + 3 + k], c = tri[9 * (int64_t)j + 6 + k];
            double lo = a < b ? a : b, hi = a > b ? a : b;
            if (c < lo) lo = c;
            if (c > hi) hi = c;
            /* widened so that the box test never culls a triangle the exact test accepts */
            double pad = 1e-9 * (fabs(lo) + fabs(hi) + 1.0);
            p[j].lo[k] = lo - pad;
            p[j].hi[k] = hi + pad;
            p[j].c[k] = 0.5 * (lo + hi);
        }
        p[j].id = j;
    }
    M->nodes = (node64 *)calloc((size_t)2 * n_tri, sizeof(node64));
    int32_t nn = 0;
    build_node(M, p, 0, n_tri, &nn);
    M->n_nodes = nn;
    M->tris = (tri64 *)malloc(sizeof(tri64) * (size_t)n_tri);
    for (int32_t i = 0; i < n_tri; i++) {
        int32_t j = p[i].id;
        const float *t = tri + 9 * (int64_t)j;
        tri64 *o = &M->tris[i];
        for (int k = 0; k < 3; k++) {
            /* .cl:1049-1053: E = K - M, F = L - M, computed here in double */
            o->m[k] = (double)t[6 + k];
            o->e[k] = (double)t[k] - (double)t[6 + k];
            o->f[k] = (double)t[3 + k] - (double)t[6 + k];
        }
        o->id = j;
    }
    free(p);
    return M;
}

void lpo64_mesh_free(lpo64_mesh *M)
{
    if (!M) return;
    free(M->tris);
    free(M->nodes);
    free(M);
}

/* The intersection of FindTriangleInPath (.cl:1049-1067) in double; updates (best, bid)
 * if the triangle is hit at 0 < t < best, or at t == best with a lower index. */
static inline void test_tri64(const tri64 *T, d3 p, d3 v, int32_t ref_tri, double *best, int32_t *bid)
{
    if (T->id == ref_tri) return;
    d3 E = mk(T->e[0], T->e[1], T->e[2]), F = mk(T->f[0], T->f[1], T->f[2]);
    d3 G = sub(p, mk(T->m[0], T->m[1], T->m[2]));
    d3 GE = cross(G, E), VF = cross(v, F);
    double w = dot(VF, E);
    double t = dot(GE, F) / w;
    double k = dot(VF, G) / w;
    double l = dot(GE, v) / w;
    if (t > 0.0 && k >= 0.0 && l >= 0.0 && (k + l) < 1.0 && (t < *best || (t == *best && T->id < *bid))) {
        *best = t;
        *bid = T->id;
    }
}

/* Nearest triangle along (p, v), t in (0, bound], t < 10000, ref_tri excluded. */
int32_t lpo64_mesh_query(const lpo64_mesh *M, int32_t ref_tri, const double pp[3], const double vv[3],
                         double bound, double *t_out)
{
    d3 p = mk(pp[0], pp[1], pp[2]), v = mk(vv[0], vv[1], vv[2]);
    double best = bound < NOHIT ? bound : NOHIT;
    /* hits at exactly `bound` count (.cl:1442: steptoboundary <= stepsize) */
    double lim_best = best;
    int32_t bid = 0x7fffffff;
    if (M->n_tri <= 0) { *t_out = NOHIT; return -1; }
    double inv[3], o[3];
    double vd[3] = {v.x, v.y, v.z}, pd[3] = {p.x, p.y, p.z};
    for (int k = 0; k < 3; k++) {
        inv[k] = 1.0 / (fabs(vd[k]) > 1e-300 ? vd[k] : copysign(1e-300, vd[k]));
        o[k] = pd[k];
    }
    int32_t stack[128];
    int sp = 0;
    stack[sp++] = 0;
    best = lim_best * (1.0 + 1e-12) + 1e-300;  /* accept t == bound in the test below */
    while (sp > 0) {
        const node64 *nd = &M->nodes[stack[--sp]];
        double tn = 0.0, tf = best;
        int miss = 0;
        for (int k = 0; k < 3 && !miss; k++) {
            double t0 = (nd->lo[k] - o[k]) * inv[k], t1 = (nd->hi[k] - o[k]) * inv[k];
            if (t0 > t1) { double s = t0; t0 = t1; t1 = s; }
            if (t0 > tn) tn = t0;
            if (t1 < tf) tf = t1;
            if (tn > tf * (1.0 + 1e-12) + 1e-12) miss = 1;
        }
        if (miss) continue;
        if (nd->left < 0) {
            for (int32_t i = nd->first; i < nd->first + nd->count; i++) test_tri64(&M->tris[i], p, v, ref_tri, &best, &bid);
        } else {
            if (sp + 2 > 128) continue;   /* cannot happen for trees of depth < 126 */
            stack[sp++] = nd->right;
            stack[sp++] = nd->left;
        }
    }
    if (bid == 0x7fffffff || !(best <= lim_best) || !(best < NOHIT)) {
        *t_out = NOHIT;
        return -1;
    }
    *t_out = best;
    return bid;
}

/* Brute-force scan in double (the reference's loop order), for checking the tree. */
int32_t lpo64_find_triangle(const float *tri, int32_t n_tri, int32_t ref_tri, const double pp[3],
                            const double vv[3], double bound, double *t_out)
{
    d3 p = mk(pp[0], pp[1], pp[2]), v = mk(vv[0], vv[1], vv[2]);
    double best = NOHIT;
    int32_t bid = -1;
    for (int32_t j = 0; j < n_tri; j++) {
        if (j == ref_tri) continue;
        const float *t = tri + 9 * (int64_t)j;
        d3 Mv = mk(t[6], t[7], t[8]);
        d3 E = sub(mk(t[0], t[1], t[2]), Mv), F = sub(mk(t[3], t[4], t[5]), Mv), G = sub(p, Mv);
        d3 GE = cross(G, E), VF = cross(v, F);
        double w = dot(VF, E);
        double tt = dot(GE, F) / w, k = dot(VF, G) / w, l = dot(GE, v) / w;
        if (tt < best && tt > 0.0 && k >= 0.0 && l >= 0.0 && (k + l) < 1.0) {
            best = tt;
            bid = j;
        }
    }
    if (bid >= 0 && !(best <= bound)) {
        bid = -1;
        best = NOHIT;
    }
    *t_out = best;
    return bid;
}

/* ------------------------------------------------------------------ RNG */
/* Draw slots of one transport event (the layout of lp_oracle.c and the CUDA path). */
enum { SLOT_STEP_ = 0, SLOT_ANGLE_ = 1, SLOT_AZIMUTH_ = 2, SLOT_ROULETTE_ = 3 };

typedef struct { uint32_t key[2], ctr[4], buf[4]; uint64_t draws; } rng64_t;

static inline void rng_photon(rng64_t *r, const lpo_problem *P, int64_t pid)
{
    r->draws = 0;
    r->key[0] = (uint32_t)P->seed;
    r->key[1] = (uint32_t)(P->seed >> 32);
    r->ctr[0] = (uint32_t)(uint64_t)pid;
    r->ctr[1] = (uint32_t)((uint64_t)pid >> 32);
    r->ctr[2] = 0;
    r->ctr[3] = P->stream;
}
static inline void rng_event(rng64_t *r, uint32_t ev)
{
    r->ctr[2] = ev;
    lpo_philox4x32_10(r->ctr, r->key, r->buf);
}
/* the 24-bit uniform of the CUDA path, ((x >> 8) | 1) * 2^-24, exactly, in double */
static inline double rng_slot(rng64_t *r, int slot)
{
    r->draws++;
    return (double)((r->buf[slot] >> 8) | 1u) * 0x1.0p-24;
}

/* ------------------------------------------------------------------ physics */
typedef struct {
    const lpo_problem *P;
    const lpo64_mesh *M;
    lpo_geometry g;
    d3 eZ, POI, nX, nY, nZ;
    double Rsp, distMin;
} ctx64_t;

/* Rspecular (.cl:273-299) in double. */
static double rspecular64(const float *nm)
{
    double n1 = nm[0], n2 = nm[4], mua1 = nm[5], mus1 = nm[6];
    double temp = (n1 - n2) / (n1 + n2);
    double r1 = temp * temp;
    if (mua1 == 0.0 && mus1 == 0.0) {
        double n3 = nm[8];
        temp = (n2 - n3) / (n2 + n3);
        double r2 = temp * temp;
        r1 = r1 + (1 - r1) * (1 - r1) * r2 / (1 - r1 * r2);
    }
    return r1;
}

/* GetFresnel (.cl:857-907) in double. */
double lpo64_fresnel(double n1, double n2, double cosIn)
{
    double r;
    if (n1 == n2) {
        r = 0.0;
    } else if (fabs(cosIn) == 1.0) {
        r = (n1 - n2) / (n1 + n2);
        r *= r;
    } else if (cosIn == 0.0) {
        r = 1.0;
    } else {
        double sinIn = sqrt(1 - cosIn * cosIn);
        double sinOut = n1 * sinIn / n2;
        if (sinOut >= 1.0) {
            r = 1.0;
        } else {
            double cosOut = sqrt(1 - sinOut * sinOut);
            double cap = cosIn * cosOut - sinIn * sinOut;
            double cam = cosIn * cosOut + sinIn * sinOut;
            double sap = sinIn * cosOut + cosIn * sinOut;
            double sam = sinIn * cosOut - cosIn * sinOut;
            r = 0.5 * (sam * sam) * ((cam * cam) + (cap * cap)) / ((sap * sap) * (cam * cam));
        }
    }
    return r;
}

static inline d3 rotate(d3 vec, d3 axis, double c, double s)
{
    /* Rotate (.cl:697-708) */
    double nDx = dot(axis, vec);
    d3 nXx = cross(axis, vec);
    d3 nXxXn = cross(nXx, axis);
    return add(add(scl(nDx, axis), scl(c, nXxXn)), scl(s, nXx));
}

/* VScatter (.cl:597-655) in double. */
static d3 vscatter64(d3 v, double g, double xt, double xp)
{
    d3 e_rot = mk(0, 0, 0);
    if (v.z != 0.0) e_rot = mk(1, 1, -(v.x + v.y) / v.z);
    else if (v.y != 0.0) e_rot = mk(1, -(v.x) / v.y, 0);
    else if (v.x != 0.0) e_rot = mk(0, 1, 0);
    e_rot = normalize(e_rot);
    double cosTheta;
    if (g != 0.0) {
        double g1 = (1 - g * g) / (1 - g + 2 * g * xt);
        cosTheta = (1 + g * g - g1 * g1) / (2 * g);
        if (cosTheta < -1) cosTheta = -1;
        else if (cosTheta > 1) cosTheta = 1;
    } else {
        cosTheta = 2 * xt - 1;
    }
    double sinTheta = sqrt(1.0 - cosTheta * cosTheta);
    double psi = 2 * PI_D * xp;
    double cosPsi = cos(psi);
    double sinPsi = sqrt(1.0 - cosPsi * cosPsi);
    if (psi > PI_D) sinPsi = -sinPsi;
    d3 rot_theta = normalize(rotate(v, e_rot, cosTheta, sinTheta));
    return normalize(rotate(rot_theta, v, cosPsi, sinPsi));
}

static inline void tadd(uint64_t *a, double w) { *a += fix64(w); }

static inline int trunc_sat(double x)
{
    if (x != x) return 0;
    if (x > 1e9) return 1000000000;
    if (x < -1e9) return -1000000000;
    return (int)x;
}
static inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

/* Absorption deposit into the r-z and voxel grids (.cl:254-271 with z rows, as lp_oracle.c). */
static void record_absorption64(const ctx64_t *C, lpo_tallies *T, d3 c, double dw, double mua)
{
    const lpo_problem *P = C->P;
    const float *dg = P->det_grid;
    double radius = sqrt(c.x * c.x + c.y * c.y) * sign_cl(c.x) / (double)dg[3];
    if (T->rz) {
        int row = (int)floor(c.z / (double)dg[2]);
        int col = (int)floor(radius + (double)C->g.dimR);
        if (row >= 0 && row < C->g.rz_nz && col >= 0 && col < C->g.rz_nr) {
            uint64_t *r = T->rz + 2 * ((int64_t)row * C->g.rz_nr + col);
            tadd(&r[0], dw);
            if (mua > 0) tadd(&r[1], dw / mua);
        } else {
            T->counters[LPO_C_RZ_DROP]++;
        }
    }
    if (T->vox && P->vox_n[0] > 0) {
        int ix = (int)floor(c.x / (double)P->vox_d[0] + 0.5 * (double)P->vox_n[0]);
        int iy = (int)floor(c.y / (double)P->vox_d[1] + 0.5 * (double)P->vox_n[1]);
        int iz = (int)floor(c.z / (double)P->vox_d[2]);
        if (ix >= 0 && ix < P->vox_n[0] && iy >= 0 && iy < P->vox_n[1] && iz >= 0 && iz < P->vox_n[2])
            tadd(&T->vox[((int64_t)iz * P->vox_n[1] + iy) * P->vox_n[0] + ix], dw);
        else
            T->counters[LPO_C_VOX_DROP]++;
    }
}

/* Exit binning of CalculatePropagation.cpp:1553-1626 plus radial bins and rings. */
static void bin_exit64(const ctx64_t *C, lpo_tallies *T, const double rec[8], const double *L, const int64_t *K)
{
    const lpo_problem *P = C->P;
    const lpo_geometry *g = &C->g;
    const float *dg = P->det_grid;
    double s = rec[3], f = rec[4], t = rec[5];
    if (s == 0.0 && f == 0.0 && t == 0.0) return;
    int hx = g->dimx / 2, hy = g->dimy / 2;
    int x = clampi(trunc_sat(rec[0] / dg[0]), -hx, hx);
    int y = clampi(trunc_sat(rec[1] / dg[1]), -hy, hy);
    uint64_t *c = T->sft + 3 * ((int64_t)(y + hy) * g->sft_nx + (x + hx));
    tadd(&c[0], s);
    tadd(&c[1], f);
    tadd(&c[2], t);
    int ai = clampi(trunc_sat(rec[6] * 180.0 / PI_D / (double)dg[5]), 0, g->dimAlpha - 1);
    int ri = clampi(trunc_sat(rec[7] / dg[3]), 0, g->dimR - 1);
    uint64_t *r = T->rtd + 3 * ((int64_t)ai * g->dimR + ri);
    tadd(&r[0], s);
    tadd(&r[1], f);
    tadd(&r[2], t);
    double rho = sqrt(rec[0] * rec[0] + rec[1] * rec[1]);
    if (T->rbins && P->n_rbins > 0) {
        int b = trunc_sat(rho / (double)P->rbin_dr);
        if (b >= 0 && b < P->n_rbins) {
            tadd(&T->rbins[2 * b], s);
            tadd(&T->rbins[2 * b + 1], t);
        }
    }
    if (T->det && s > 0.0) {
        for (int d = 0; d < P->n_det; d++) {
            if (rho >= (double)P->det_r[2 * d] && rho < (double)P->det_r[2 * d + 1]) {
                tadd(&T->det[2 * d], s);
                tadd(&T->det[2 * d + 1], s * s);
                if (T->grad && L) {
                    for (int rr = 0; rr < P->n_media; rr++) {
                        double a = s * L[rr], b = s * (double)K[rr];
                        double *gg = T->grad + 5 * ((int64_t)d * P->n_media + rr);
                        gg[0] += a;
                        gg[1] += b;
                        gg[2] += a * a;
                        gg[3] += b * b;
                        gg[4] += a * b;
                    }
                }
            }
        }
    }
}

/* One photon history (.cl:1287-1597) in double. */
static void trace64(const ctx64_t *C, rng64_t *R, int64_t pid, lpo_tallies *T, float *rec_out)
{
    const lpo_problem *P = C->P;
    const float *nm = P->nmuasg;
    rng_photon(R, P, pid);
    d3 v = mk(P->v_start[0], P->v_start[1], P->v_start[2]);
    d3 p = mk(P->p_start[0], P->p_start[1], P->p_start[2]);
    if (P->src_type == 1) {
        /* fibre source, event 0 (as lp_oracle.c) */
        rng_event(R, 0);
        double x1 = rng_slot(R, 0), x2 = rng_slot(R, 1), x3 = rng_slot(R, 2), x4 = rng_slot(R, 3);
        double r = (double)P->src_radius * sqrt(x1);
        double phi = 2 * PI_D * x2;
        p = add(p, add(scl(r * cos(phi), C->nX), scl(r * sin(phi), C->nY)));
        double ct = 1.0 - x3 * (1.0 - (double)P->src_cos_max);
        double stt = sqrt(1.0 - ct * ct);
        double psi = 2 * PI_D * x4;
        v = normalize(add(scl(ct, C->nZ), add(scl(stt * cos(psi), C->nX), scl(stt * sin(psi), C->nY))));
    }
    const double exit_scale = (P->compat & LPO_COMPAT_EXIT_RSP) ? (1.0 - C->Rsp) : 1.0;
    double w = 1.0 - C->Rsp, unfin = 0.0, absorbed;
    d3 SFT = mk(0, 0, 0);
    int fetal = 0, refTri = -1, curr = 0, roulette = 1;
    d3 nv = mk(0, 0, -1);
    int64_t steps = 0;
    uint64_t region_acc = 0;
    double L[LPO_MAX_MEDIA];
    int64_t K[LPO_MAX_MEDIA];
    const int track = T->grad != NULL && P->n_media <= LPO_MAX_MEDIA;
    if (track) {
        memset(L, 0, sizeof L);
        memset(K, 0, sizeof K);
    }
    do {
        rng_event(R, (uint32_t)(steps + 1));
        const float *cur = nm + 4 * curr;
        const double mua = cur[1], mus = cur[2], mut = mua + mus;
        double step;
        const int ambient = (mua == 0.0 && mus == 0.0);
        if (ambient) step = NOHIT;
        else if (unfin == 0.0) step = -log(rng_slot(R, SLOT_STEP_)) * (double)P->factor / mut;
        else {
            step = unfin / mut;
            unfin = 0.0;
        }
        double pp[3] = {p.x, p.y, p.z}, vv[3] = {v.x, v.y, v.z};
        double thit;
        int32_t tri = lpo64_mesh_query(C->M, refTri, pp, vv, step, &thit);
        T->counters[LPO_C_QUERY]++;
        if (ambient) step = thit;
        if (thit <= step) {
            T->counters[LPO_C_BOUNDARY]++;
            p = add(p, scl(thit, v));
            refTri = -1;
            double xi = rng_slot(R, SLOT_ANGLE_);
            if (tri < 0) {
                T->counters[LPO_C_MISS]++;
                w = 0;
            } else {
                if (track) L[curr] += thit;
                int inner = P->med[2 * tri], outer = P->med[2 * tri + 1];
                if (curr != inner && curr != outer) T->counters[LPO_C_MISMATCH]++;
                nv = normalize(ldf3(P->nrm, tri));
                const float *nxt = (curr == outer) ? nm + 4 * inner : nm + 4 * outer;
                if (P->compat & LPO_COMPAT_AXIS_NORMAL) {
                    if (sqrt(p.x * p.x + p.y * p.y) < 0.01) nv = scl(sign_cl(dot(nv, C->eZ)), C->nZ);
                }
                /* TransmitOrReflect (.cl:921-1018) */
                double cosIn = dot(nv, v), n1 = cur[0], n2 = nxt[0];
                double cos_crit = 0.0;
                if (n1 > n2) cos_crit = sqrt(1.0 - (n2 / n1) * (n2 / n1));
                double rf;
                if (fabs(cosIn) <= cos_crit) rf = 1.0;
                else rf = lpo64_fresnel(n1, n2, (P->compat & LPO_COMPAT_SIGNED_FRESNEL) ? cosIn : fabs(cosIn));
                d3 e_y = normalize(cross(nv, cross(nv, v)));
                int newID;
                double muaNew, musNew;
                if (xi > rf) {
                    double sinT = sqrt(1 - cosIn * cosIn) * n1 / n2;
                    double cosT = -sqrt(1 - sinT * sinT);
                    if (cosIn > 0.0) cosT = fabs(cosT);
                    v = normalize(sub(scl(cosT, nv), scl(sinT, e_y)));
                    newID = (cosIn > 0) ? outer : inner;
                    muaNew = nxt[1];
                    musNew = nxt[2];
                } else {
                    double sinR = sqrt(1 - cosIn * cosIn);
                    v = neg(normalize(add(scl(cosIn, nv), scl(sinR, e_y))));
                    newID = curr;
                    muaNew = mua;
                    musNew = mus;
                }
                if (muaNew == 0 || musNew == 0) {
                    SFT.y = 0;
                    double dist = fabs(dot(C->nZ, sub(p, C->POI)));
                    if (dist > C->distMin) {
                        SFT.z = w * exit_scale;
                    } else {
                        if (fetal) SFT.y = w * exit_scale;
                        SFT.x = w * exit_scale;
                    }
                    w = 0;
                }
                int prev = curr;
                curr = newID;
                refTri = tri;
                if (curr == P->fetal_id) fetal = 1;
                unfin = (step - thit) * mut;
                if (curr != prev && T->region) {
                    T->region[prev] += region_acc;
                    region_acc = 0;
                }
            }
        } else {
            T->counters[LPO_C_SCATTER]++;
            p = add(p, scl(step, v));
            refTri = -1;
            if (track) {
                L[curr] += step;
                K[curr]++;
            }
            absorbed = 0.0;
            if (mua > 0.0 && mus > 0.0) {
                absorbed = w * (mua / mut);
                w -= absorbed;
            }
            double xt = rng_slot(R, SLOT_ANGLE_), xp = rng_slot(R, SLOT_AZIMUTH_);
            v = vscatter64(v, (double)cur[3], xt, xp);
            d3 pr = sub(p, C->POI);
            d3 co = mk(dot(C->nX, pr), dot(C->nY, pr), dot(C->nZ, pr));
            record_absorption64(C, T, co, absorbed, mua);
            region_acc += fix64(absorbed);
        }
        if (w < (double)P->w_threshold && w > 0.0) {
            double xi = rng_slot(R, SLOT_ROULETTE_);
            T->counters[LPO_C_ROULETTE]++;
            if (xi < (double)P->chance) {
                w /= (double)P->chance;
                roulette = 1;
            } else {
                w = 0;
                roulette = 0;
            }
        }
        steps++;
        if (P->max_steps > 0 && steps >= P->max_steps && w > 0.0) {
            T->counters[LPO_C_CAPPED]++;
            w = 0;
        }
    } while (w > 0.0 && (w > (double)P->w_threshold || roulette));
    if (T->region) T->region[curr] += region_acc;
    T->counters[LPO_C_PHOTONS]++;
    T->counters[LPO_C_DRAWS] += R->draws;
    /* exit record (.cl:1583-1594) */
    double rec[8];
    double cs = dot(v, nv);
    if (cs > 1.0) cs = 1.0;
    if (cs < -1.0) cs = -1.0;
    d3 d = sub(C->POI, p), pr = sub(p, C->POI);
    rec[0] = dot(C->nX, pr);
    rec[1] = dot(C->nY, pr);
    rec[2] = dot(C->nZ, pr);
    rec[3] = SFT.x;
    rec[4] = SFT.y;
    rec[5] = SFT.z;
    rec[6] = fabs(acos(cs));
    rec[7] = sqrt(dot(d, d));
    if (rec_out)
        for (int k = 0; k < 8; k++) rec_out[k] = (float)rec[k];
    bin_exit64(C, T, rec, track ? L : NULL, track ? K : NULL);
}

/* ------------------------------------------------------------------ driver */
typedef struct {
    const ctx64_t *C;
    int64_t first, n, chunk;
    int64_t *next;
    pthread_mutex_t *lock;
    lpo_tallies T;
    float *exit_rec;
} worker64_t;

static void *worker64(void *arg)
{
    worker64_t *W = (worker64_t *)arg;
    rng64_t R;
    memset(&R, 0, sizeof R);
    for (;;) {
        int64_t s;
        pthread_mutex_lock(W->lock);
        s = *W->next;
        *W->next += W->chunk;
        pthread_mutex_unlock(W->lock);
        if (s >= W->n) break;
        int64_t e = s + W->chunk < W->n ? s + W->chunk : W->n;
        for (int64_t i = s; i < e; i++)
            trace64(W->C, &R, W->first + i, &W->T, W->exit_rec ? W->exit_rec + 8 * i : NULL);
    }
    return NULL;
}

static void merge64(uint64_t *dst, const uint64_t *src, size_t n)
{
    if (!dst || !src) return;
    for (size_t i = 0; i < n; i++) dst[i] += src[i];
}

int lpo64_run(const lpo_problem *P, const lpo64_mesh *mesh, int64_t first, int64_t n, int nthreads,
              lpo_tallies *T)
{
    if (P->rng_mode != LPO_RNG_PHILOX || P->n_media > LPO_MAX_MEDIA) return 1;
    ctx64_t C;
    C.P = P;
    lpo64_mesh *own = NULL;
    if (!mesh) mesh = own = lpo64_mesh_build(P->tri, P->n_tri);
    C.M = mesh;
    lpo_geometry_of(P->dimensions, P->det_grid, &C.g);
    C.POI = mk(P->ep0xyz[0], P->ep0xyz[1], P->ep0xyz[2]);
    C.eZ = mk(P->ep0xyz[9], P->ep0xyz[10], P->ep0xyz[11]);
    C.nX = normalize(mk(P->ep0xyz[3], P->ep0xyz[4], P->ep0xyz[5]));
    C.nY = normalize(mk(P->ep0xyz[6], P->ep0xyz[7], P->ep0xyz[8]));
    C.nZ = normalize(C.eZ);
    C.Rsp = rspecular64(P->nmuasg);
    C.distMin = (double)P->det_grid[2] * (double)C.g.dimz / 2.0;   /* .cl:1351 */
    if (n <= 0) {
        lpo64_mesh_free(own);
        return 0;
    }
    if (nthreads <= 0) nthreads = (int)sysconf(_SC_NPROCESSORS_ONLN);
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    const lpo_geometry *g = &C.g;
    const size_t nsft = (size_t)g->sft_nx * g->sft_ny * 3, nrtd = (size_t)g->dimR * g->dimAlpha * 3;
    const size_t nrz = (size_t)g->rz_nr * g->rz_nz * 2;
    const size_t nvox = P->vox_n[0] > 0 ? (size_t)P->vox_n[0] * P->vox_n[1] * P->vox_n[2] : 0;
    const size_t ngrad = (size_t)(P->n_det > 0 ? P->n_det : 0) * P->n_media * 5;
    int64_t next = 0;
    pthread_mutex_t lock = PTHREAD_MUTEX_INITIALIZER;
    worker64_t *W = (worker64_t *)calloc((size_t)nthreads, sizeof(worker64_t));
    pthread_t *th = (pthread_t *)calloc((size_t)nthreads, sizeof(pthread_t));
    int64_t chunk = n / ((int64_t)nthreads * 16);
    if (chunk < 1) chunk = 1;
    if (chunk > 4096) chunk = 4096;
    for (int t = 0; t < nthreads; t++) {
        worker64_t *w = &W[t];
        w->C = &C;
        w->first = first;
        w->n = n;
        w->chunk = chunk;
        w->next = &next;
        w->lock = &lock;
        w->exit_rec = T->exit_rec;
        w->T.sft = T->sft ? (uint64_t *)calloc(nsft, 8) : NULL;
        w->T.rtd = T->rtd ? (uint64_t *)calloc(nrtd, 8) : NULL;
        w->T.rz = T->rz ? (uint64_t *)calloc(nrz, 8) : NULL;
        w->T.vox = (T->vox && nvox) ? (uint64_t *)calloc(nvox, 8) : NULL;
        w->T.rbins = (T->rbins && P->n_rbins > 0) ? (uint64_t *)calloc((size_t)P->n_rbins * 2, 8) : NULL;
        w->T.region = T->region ? (uint64_t *)calloc((size_t)P->n_media, 8) : NULL;
        w->T.det = (T->det && P->n_det > 0) ? (uint64_t *)calloc((size_t)P->n_det * 2, 8) : NULL;
        w->T.grad = (T->grad && ngrad) ? (double *)calloc(ngrad, 8) : NULL;
        if (t > 0) pthread_create(&th[t], NULL, worker64, w);
    }
    worker64(&W[0]);
    for (int t = 1; t < nthreads; t++) pthread_join(th[t], NULL);
    for (int t = 0; t < nthreads; t++) {
        worker64_t *w = &W[t];
        merge64(T->sft, w->T.sft, nsft);
        merge64(T->rtd, w->T.rtd, nrtd);
        merge64(T->rz, w->T.rz, nrz);
        merge64(T->vox, w->T.vox, nvox);
        merge64(T->rbins, w->T.rbins, (size_t)(P->n_rbins > 0 ? P->n_rbins : 0) * 2);
        merge64(T->region, w->T.region, (size_t)P->n_media);
        merge64(T->det, w->T.det, (size_t)(P->n_det > 0 ? P->n_det : 0) * 2);
        if (T->grad && w->T.grad)
            for (size_t k = 0; k < ngrad; k++) T->grad[k] += w->T.grad[k];
        for (int k = 0; k < LPO_NCOUNTERS; k++) T->counters[k] += w->T.counters[k];
        free(w->T.sft); free(w->T.rtd); free(w->T.rz); free(w->T.vox);
        free(w->T.rbins); free(w->T.region); free(w->T.det); free(w->T.grad);
    }
    free(W);
    free(th);
    lpo64_mesh_free(own);
    return 0;
}
