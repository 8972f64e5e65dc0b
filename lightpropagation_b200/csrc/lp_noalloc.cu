// lp_noalloc.cu -- lp_run_noalloc: photon transport without any device allocation.
//
// Some callers cannot let a library call cudaMalloc: an application whose device memory
// comes from its own arena with a fixed budget, or code that cannot afford the
// device-wide synchronisation that cudaFree implies.  This entry point gives them the transport with all
// scratch in the file-scope array below, so it allocates nothing; the caller passes
// the mesh and the output tallies in its own device memory.
//
// Scratch layout (offsets below): photon work counter and event counters (cleared at
// every call), the media table, and a small BVH built on the device from the caller's
// reference-layout mesh arrays (leaves of 4 triangles in input order, a heap-ordered
// binary tree over them).  The transport itself is the existing reference-arithmetic
// kernel, launched with pointers into this array; its results equal those of lp_run
// in reference-arithmetic mode for the same seed and photon range.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>

#include "../../include/lpcuda.h"
#include "lp_kernel.cuh"

namespace lp {
int smem_bytes(int nodes_smem, int tris_smem);
cudaError_t launch_transport_exact(const KParams &P, int grid, int smem, cudaStream_t s);
cudaError_t transport_occupancy_exact(int smem, int *blocks_per_sm);
void set_thread_error(const char *msg);
float rspecular_of(const float *nmuasg, int n_media);
std::mutex &launch_mutex();
}  // namespace lp

namespace {
using namespace lp;

constexpr int kLeafTris = 4;
constexpr int kMaxLeaves = (LP_NOALLOC_MAX_TRI + kLeafTris - 1) / kLeafTris;
constexpr int kMaxNodes = kMaxLeaves;
constexpr size_t OFF_WORK = 0;
constexpr size_t OFF_CNT = 8;                       // 16 counters -> 136 bytes used
// set as the work counter when the mesh fails the device-side check: every photon index
// handed out is then past the range, so the transport kernel traces nothing
constexpr unsigned long long kRejectAll = 1ull << 62;
constexpr size_t HEADER = 256;                      // cleared at every call
constexpr size_t OFF_MEDIA = HEADER;
constexpr size_t OFF_NODE_A = OFF_MEDIA + LP_NOALLOC_MAX_MEDIA * sizeof(Medium);
constexpr size_t OFF_NODE_B = OFF_NODE_A + kMaxNodes * 16;
constexpr size_t OFF_NODE_C = OFF_NODE_B + kMaxNodes * 16;
constexpr size_t OFF_NODE_D = OFF_NODE_C + kMaxNodes * 16;
constexpr size_t OFF_TRI_A = OFF_NODE_D + kMaxNodes * 16;
constexpr size_t OFF_TRI_B = OFF_TRI_A + LP_NOALLOC_MAX_TRI * 16;
constexpr size_t OFF_TRI_C = OFF_TRI_B + LP_NOALLOC_MAX_TRI * 16;
constexpr size_t OFF_ATTR = OFF_TRI_C + LP_NOALLOC_MAX_TRI * 16;
constexpr size_t OFF_BOX = OFF_ATTR + LP_NOALLOC_MAX_TRI * 16;   // leaf and node boxes, 6 floats each
constexpr size_t OFF_END = OFF_BOX + (size_t)(kMaxLeaves + kMaxNodes) * 24;
static_assert(OFF_END <= LP_NOALLOC_SCRATCH_BYTES, "scratch layout exceeds the static array");
static_assert(OFF_NODE_A % 16 == 0 && OFF_TRI_A % 16 == 0 && OFF_ATTR % 16 == 0, "float4 alignment");

static __device__ __align__(256) unsigned char g_noalloc_scratch[LP_NOALLOC_SCRATCH_BYTES];

struct MediaParams {
    int32_t n;
    float4 v[LP_NOALLOC_MAX_MEDIA];
};

__device__ __forceinline__ void grow(float *b, float x, float y, float z)
{
    b[0] = fminf(b[0], x); b[1] = fminf(b[1], y); b[2] = fminf(b[2], z);
    b[3] = fmaxf(b[3], x); b[4] = fmaxf(b[4], y); b[5] = fmaxf(b[5], z);
}

// One block: media table, triangles in the kernel's SoA layout, per-triangle attributes
// and the BVH.  Explicit round-to-nearest intrinsics reproduce the host's IEEE values
// (no contraction), so the transport sees exactly the inputs lp_set_* would produce.
__global__ void __launch_bounds__(256) noalloc_setup_kernel(const float *tri, const float *nrm, const int32_t *med,
                                                            int n_tri, const __grid_constant__ MediaParams mp,
                                                            unsigned char *s)
{
    Medium *media = reinterpret_cast<Medium *>(s + OFF_MEDIA);
    float4 *na = reinterpret_cast<float4 *>(s + OFF_NODE_A), *nb = reinterpret_cast<float4 *>(s + OFF_NODE_B);
    float4 *nc = reinterpret_cast<float4 *>(s + OFF_NODE_C);
    int4 *nd = reinterpret_cast<int4 *>(s + OFF_NODE_D);
    float4 *ta = reinterpret_cast<float4 *>(s + OFF_TRI_A), *tb = reinterpret_cast<float4 *>(s + OFF_TRI_B);
    float4 *tc = reinterpret_cast<float4 *>(s + OFF_TRI_C), *at = reinterpret_cast<float4 *>(s + OFF_ATTR);
    float *box = reinterpret_cast<float *>(s + OFF_BOX);
    const int tid = threadIdx.x, bd = blockDim.x;
    for (int i = tid; i < mp.n; i += bd) {
        const float4 q = mp.v[i];
        Medium m;
        m.n = q.x; m.mua = q.y; m.mus = q.z; m.g = q.w;
        m.mut = __fadd_rn(q.y, q.z);
        m.alb = __fdiv_rn(q.y, m.mut);
        m.absorbs = (q.y > 0.0f && q.z > 0.0f) ? 1 : 0;
        m.ambient = (q.y == 0.0f && q.z == 0.0f) ? 1 : 0;
        m.inv_mut = m.mut > 0.0f ? __fdiv_rn(1.0f, m.mut) : 0.0f;
        m.inv_mua = q.y > 0.0f ? __fdiv_rn(1.0f, q.y) : 0.0f;
        m.hg_a = __fsub_rn(1.0f, __fmul_rn(q.w, q.w));
        m.hg_b = __fsub_rn(1.0f, q.w);
        m.hg_c = __fmul_rn(2.0f, q.w);
        m.hg_d = __fadd_rn(1.0f, __fmul_rn(q.w, q.w));
        m.hg_inv2g = q.w != 0.0f ? __fdiv_rn(1.0f, __fmul_rn(2.0f, q.w)) : 0.0f;
        m.pad_ = 0.0f;
        media[i] = m;
    }
    __shared__ float s_b[6][256];
    __shared__ float s_abs[256];
    float b[6] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY};
    float amax = 0.0f;
    for (int j = tid; j < n_tri; j += bd) {
        const float *t = tri + 9 * (int64_t)j;
        const float Ex = __fsub_rn(t[0], t[6]), Ey = __fsub_rn(t[1], t[7]), Ez = __fsub_rn(t[2], t[8]);
        const float Fx = __fsub_rn(t[3], t[6]), Fy = __fsub_rn(t[4], t[7]), Fz = __fsub_rn(t[5], t[8]);
        ta[j] = make_float4(t[6], t[7], t[8], Ex);
        tb[j] = make_float4(Ey, Ez, Fx, Fy);
        tc[j] = make_float4(Fz, __int_as_float(j), 0.0f, 0.0f);
        float x = nrm[3 * (int64_t)j], y = nrm[3 * (int64_t)j + 1], z = nrm[3 * (int64_t)j + 2];
        const float l = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(x, x), __fmul_rn(y, y)), __fmul_rn(z, z)));
        if (l != 0.0f) {
            x = __fdiv_rn(x, l);
            y = __fdiv_rn(y, l);
            z = __fdiv_rn(z, l);
        }
        const int in_id = med[2 * (int64_t)j], out_id = med[2 * (int64_t)j + 1];
        if (in_id < 0 || in_id >= mp.n || out_id < 0 || out_id >= mp.n) {
            // lp_set_mesh rejects such an id; here the mesh lives in device memory, so the
            // check is made on the device: the triangle is counted and nothing is traced
            atomicAdd(reinterpret_cast<unsigned long long *>(s + OFF_CNT) + LP_C_BAD_INPUT, 1ull);
        }
        const int inner = min(max(in_id, 0), mp.n - 1);
        const int outer = min(max(out_id, 0), mp.n - 1);
        at[j] = make_float4(x, y, z, __int_as_float(inner | (outer << 16)));
        for (int k = 0; k < 9; ++k) amax = fmaxf(amax, fabsf(t[k]));
        for (int v = 0; v < 3; ++v) grow(b, t[3 * v], t[3 * v + 1], t[3 * v + 2]);
    }
    for (int k = 0; k < 6; ++k) s_b[k][tid] = b[k];
    s_abs[tid] = amax;
    __syncthreads();
    for (int o = bd / 2; o > 0; o >>= 1) {
        if (tid < o) {
            for (int k = 0; k < 3; ++k) s_b[k][tid] = fminf(s_b[k][tid], s_b[k][tid + o]);
            for (int k = 3; k < 6; ++k) s_b[k][tid] = fmaxf(s_b[k][tid], s_b[k][tid + o]);
            s_abs[tid] = fmaxf(s_abs[tid], s_abs[tid + o]);
        }
        __syncthreads();
    }
    const float ext = fmaxf(fmaxf(s_b[3][0] - s_b[0][0], s_b[4][0] - s_b[1][0]), s_b[5][0] - s_b[2][0]);
    const float margin = 1e-5f * fmaxf(ext, s_abs[0]) + 1e-30f;
    // leaf boxes
    const int L = (n_tri + kLeafTris - 1) / kLeafTris;
    for (int leaf = tid; leaf < L; leaf += bd) {
        float lb[6] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY};
        for (int j = kLeafTris * leaf; j < min(kLeafTris * (leaf + 1), n_tri); ++j)
            for (int v = 0; v < 3; ++v) {
                const float *p = tri + 9 * (int64_t)j + 3 * v;
                grow(lb, p[0], p[1], p[2]);
            }
        for (int k = 0; k < 6; ++k) box[6 * leaf + k] = lb[k];
    }
    __syncthreads();
    // internal boxes, bottom-up in heap order: node k has children 2k+1, 2k+2; heap
    // positions >= L-1 are leaves (leaf index = position - (L-1))
    const int NI = L > 1 ? L - 1 : 1;
    float *ib = box + 6 * kMaxLeaves;
    if (tid == 0 && L > 1) {
        for (int k = L - 2; k >= 0; --k) {
            for (int q = 0; q < 6; ++q) ib[6 * k + q] = (q < 3) ? INFINITY : -INFINITY;
            for (int c = 2 * k + 1; c <= 2 * k + 2; ++c) {
                const float *cb = (c >= L - 1) ? box + 6 * (c - (L - 1)) : ib + 6 * c;
                for (int q = 0; q < 3; ++q) ib[6 * k + q] = fminf(ib[6 * k + q], cb[q]);
                for (int q = 3; q < 6; ++q) ib[6 * k + q] = fmaxf(ib[6 * k + q], cb[q]);
            }
        }
    }
    __syncthreads();
    for (int k = tid; k < NI; k += bd) {
        float cbx[2][6];
        int ref[2];
        for (int s2 = 0; s2 < 2; ++s2) {
            const int c = (L > 1) ? 2 * k + 1 + s2 : 0;   // a single leaf is both children of the root
            const bool leaf = (L == 1) || c >= L - 1;
            const int li = (L == 1) ? 0 : c - (L - 1);
            const float *src = leaf ? box + 6 * li : ib + 6 * c;
            for (int q = 0; q < 3; ++q) cbx[s2][q] = src[q] - margin;
            for (int q = 3; q < 6; ++q) cbx[s2][q] = src[q] + margin;
            if (leaf) {
                const int first = kLeafTris * li, cnt = min(kLeafTris, n_tri - first);
                ref[s2] = ~((first << 3) | (cnt - 1));
            } else {
                ref[s2] = c;
            }
        }
        na[k] = make_float4(cbx[0][0], cbx[0][3], cbx[0][1], cbx[0][4]);
        nb[k] = make_float4(cbx[1][0], cbx[1][3], cbx[1][1], cbx[1][4]);
        nc[k] = make_float4(cbx[0][2], cbx[0][5], cbx[1][2], cbx[1][5]);
        nd[k] = make_int4(ref[0], ref[1], 0, 0);
    }
    __syncthreads();
    if (tid == 0 && reinterpret_cast<unsigned long long *>(s + OFF_CNT)[LP_C_BAD_INPUT] != 0)
        *reinterpret_cast<unsigned long long *>(s + OFF_WORK) = kRejectAll;
}

std::mutex g_mu;
void *g_scratch_addr[256] = {};

// The device address of the scratch array on the current device.  Outside stream
// capture it is looked up again at every call (cheap), so a module reloaded after
// cudaDeviceReset is followed; inside a capture the address cached by an earlier call
// on this device is used, because the lookup may not be captured.
int scratch_address(int dev, cudaStream_t s, void **out)
{
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) != cudaSuccess) cs = cudaStreamCaptureStatusNone;
    std::lock_guard<std::mutex> lk(g_mu);
    if (cs == cudaStreamCaptureStatusNone || !g_scratch_addr[dev]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return LP_ERR_CUDA;
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
    return LP_OK;
}

int reject(int code, const char *msg)
{
    lp::set_thread_error(msg);
    return code;
}

float norm_component(const float *v, int k)
{
    const float l = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    return l != 0.0f ? v[k] / l : v[k];
}

}  // namespace

extern "C" int lp_run_noalloc(const lp_noalloc_args *a, void *stream)
{
    if (!a) return reject(LP_ERR_INVALID, "lp_run_noalloc: args is NULL");
    if (!a->tri || !a->nrm || !a->med || !a->nmuasg || !a->sft || !a->rtd || !a->rz || !a->region)
        return reject(LP_ERR_INVALID, "lp_run_noalloc: a mesh, media or output pointer is NULL");
    if (a->n_tri < 1 || a->n_tri > LP_NOALLOC_MAX_TRI)
        return reject(LP_ERR_RANGE, "lp_run_noalloc: n_tri must be 1..LP_NOALLOC_MAX_TRI (4096)");
    if (a->n_media < 1 || a->n_media > LP_NOALLOC_MAX_MEDIA)
        return reject(LP_ERR_RANGE, "lp_run_noalloc: n_media must be 1..LP_NOALLOC_MAX_MEDIA (64)");
    if (a->n_photons < 0 || a->first < 0) return reject(LP_ERR_INVALID, "lp_run_noalloc: negative photon range");
    if (a->n_photons > lp::kMaxLaunchPhotons)
        return reject(LP_ERR_RANGE, "lp_run_noalloc: more than 2^31 photons in one call");
    if (!(a->chance > 0.0f && a->chance <= 1.0f) || !(a->factor > 0.0f) || !(a->w_threshold >= 0.0f))
        return reject(LP_ERR_INVALID, "lp_run_noalloc: bad chance, factor or weight threshold");
    for (int i = 0; i < 6; ++i)
        if (!(a->det_grid[i] > 0.0f)) return reject(LP_ERR_INVALID, "lp_run_noalloc: detection grid step not positive");
    for (int i = 0; i < 4 * a->n_media; ++i)
        if (!std::isfinite(a->nmuasg[i])) return reject(LP_ERR_INVALID, "lp_run_noalloc: non-finite optical property");
    for (int i = 0; i < 3; ++i)
        if (!(std::isfinite(a->dimensions[i]) && a->dimensions[i] > 0.0f))
            return reject(LP_ERR_INVALID, "lp_run_noalloc: model dimensions must be finite and positive");
    // tally-image extents (CalculatePropagation::InitLogVectors, CP.cpp:127-131), bounded
    // in double before the int casts: the kernel indexes the caller's sft, rtd and rz
    // buffers with them, and their sizes cannot be checked here
    const double kMaxExtent = double(1 << 20);
    for (int i = 0; i < 3; ++i)
        if (!((double)a->dimensions[i] / (double)a->det_grid[i] < kMaxExtent))
            return reject(LP_ERR_RANGE, "lp_run_noalloc: image extent beyond 2^20 cells");
    if (!(90.0 / (double)a->det_grid[5] < kMaxExtent)) return reject(LP_ERR_RANGE, "lp_run_noalloc: angle bins beyond 2^20");
    const int dimx = (int)(a->dimensions[0] / a->det_grid[0]), dimy = (int)(a->dimensions[1] / a->det_grid[1]);
    const int dimz = (int)(a->dimensions[2] / a->det_grid[2]), dimAlpha = (int)(90 / a->det_grid[5]);
    const int dimR = (int)std::ceil(std::sqrt(std::pow((double)(dimx / 2), 2) + std::pow((double)(dimy / 2), 2)));
    if (dimx < 0 || dimy < 0 || dimz < 0 || dimAlpha < 1 || dimR < 1)
        return reject(LP_ERR_RANGE, "lp_run_noalloc: image extents out of range");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= 256) return reject(LP_ERR_CUDA, "lp_run_noalloc: no current CUDA device");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // the scratch array's device address on this device (its name is only a host-side
    // stand-in in host code)
    void *base = nullptr;
    if (scratch_address(dev, s, &base) != LP_OK) return reject(LP_ERR_CUDA, "lp_run_noalloc: cudaGetSymbolAddress failed");
    if (a->n_photons == 0) return LP_OK;
    unsigned char *sb = static_cast<unsigned char *>(base);

    if ((e = cudaMemsetAsync(sb, 0, HEADER, s)) != cudaSuccess) return reject(LP_ERR_CUDA, "lp_run_noalloc: memset");
    MediaParams mp;
    std::memset(&mp, 0, sizeof mp);
    mp.n = a->n_media;
    for (int i = 0; i < a->n_media; ++i)
        mp.v[i] = make_float4(a->nmuasg[4 * i], a->nmuasg[4 * i + 1], a->nmuasg[4 * i + 2], a->nmuasg[4 * i + 3]);
    noalloc_setup_kernel<<<1, 256, 0, s>>>(a->tri, a->nrm, a->med, (int)a->n_tri, mp, sb);
    if ((e = cudaGetLastError()) != cudaSuccess) return reject(LP_ERR_CUDA, "lp_run_noalloc: setup launch");

    KParams P;
    std::memset(&P, 0, sizeof P);
    const int L = (int)((a->n_tri + kLeafTris - 1) / kLeafTris), NI = L > 1 ? L - 1 : 1;
    P.node_a = reinterpret_cast<const float4 *>(sb + OFF_NODE_A);
    P.node_b = reinterpret_cast<const float4 *>(sb + OFF_NODE_B);
    P.node_c = reinterpret_cast<const float4 *>(sb + OFF_NODE_C);
    P.node_d = reinterpret_cast<const int4 *>(sb + OFF_NODE_D);
    P.tri_a = reinterpret_cast<const float4 *>(sb + OFF_TRI_A);
    P.tri_b = reinterpret_cast<const float4 *>(sb + OFF_TRI_B);
    P.tri_c = reinterpret_cast<const float4 *>(sb + OFF_TRI_C);
    P.tri_attr = reinterpret_cast<const float4 *>(sb + OFF_ATTR);
    P.n_nodes = NI;
    P.n_tri = (int32_t)a->n_tri;
    const int base_smem = smem_bytes(0, 0);
    int room = 64 * 1024 - base_smem;
    P.nodes_smem = std::min(NI, room / 64);
    room -= P.nodes_smem * 64;
    P.tris_smem = std::min((int)a->n_tri, room / 48);
    P.media = reinterpret_cast<const Medium *>(sb + OFF_MEDIA);
    P.n_media = a->n_media;
    P.p0x = a->p_start[0]; P.p0y = a->p_start[1]; P.p0z = a->p_start[2];
    P.v0x = a->v_start[0]; P.v0y = a->v_start[1]; P.v0z = a->v_start[2];
    P.poix = a->ep0xyz[0]; P.poiy = a->ep0xyz[1]; P.poiz = a->ep0xyz[2];
    P.ezx = a->ep0xyz[9]; P.ezy = a->ep0xyz[10]; P.ezz = a->ep0xyz[11];
    P.nxx = norm_component(a->ep0xyz + 3, 0); P.nxy = norm_component(a->ep0xyz + 3, 1); P.nxz = norm_component(a->ep0xyz + 3, 2);
    P.nyx = norm_component(a->ep0xyz + 6, 0); P.nyy = norm_component(a->ep0xyz + 6, 1); P.nyz = norm_component(a->ep0xyz + 6, 2);
    P.nzx = norm_component(a->ep0xyz + 9, 0); P.nzy = norm_component(a->ep0xyz + 9, 1); P.nzz = norm_component(a->ep0xyz + 9, 2);
    P.Rsp = lp::rspecular_of(a->nmuasg, a->n_media);
    P.w0 = 1.0f - P.Rsp;
    P.exitScale = (a->compat & LP_COMPAT_EXIT_RSP) ? (1 - P.Rsp) : 1.0f;
    P.distMin = a->det_grid[2] * (float)dimz / 2.0f;
    P.src_type = (a->fiber_radius > 0.0f || a->fiber_cos_max < 1.0f) ? 1 : 0;
    P.src_radius = a->fiber_radius;
    P.src_cos_max = a->fiber_cos_max;
    P.chance = a->chance;
    P.w_th = a->w_threshold;
    P.factor = a->factor;
    P.fetal_id = a->fetal_id;
    P.compat = a->compat & LP_COMPAT_ALL;
    P.key0 = (uint32_t)a->seed;
    P.key1 = (uint32_t)(a->seed >> 32);
    P.first = a->first;
    P.n = a->n_photons;
    P.max_steps = LP_NOALLOC_MAX_STEPS;
    P.hx = dimx / 2; P.hy = dimy / 2; P.sft_nx = 2 * (dimx / 2) + 1;
    P.dimR = dimR; P.dimAlpha = dimAlpha; P.rz_nr = 2 * dimR + 1; P.rz_nz = dimz + 1;
    for (int i = 0; i < 6; ++i) P.dg[i] = a->det_grid[i];
    P.inv_dr = 1.0f / a->det_grid[3];
    P.inv_dz = 1.0f / a->det_grid[2];
    P.inv_vdx = P.inv_vdy = P.inv_vdz = 1.0f;
    P.sft = reinterpret_cast<unsigned long long *>(a->sft);
    P.rtd = reinterpret_cast<unsigned long long *>(a->rtd);
    P.rz = reinterpret_cast<unsigned long long *>(a->rz);
    P.region = reinterpret_cast<unsigned long long *>(a->region);
    P.counters = reinterpret_cast<unsigned long long *>(sb + OFF_CNT);
    P.work = reinterpret_cast<unsigned long long *>(sb + OFF_WORK);
    // voxel grid, radial bins, rings, exit records and the safety grid stay off
    const int smem = smem_bytes(P.nodes_smem, P.tris_smem);
    int per_sm = 0, sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    {
        // the kernel's shared-memory attribute is process-wide: lp_run on another thread
        // sets it too, so the setting and the launch are made under the same lock
        std::lock_guard<std::mutex> lk(lp::launch_mutex());
        if ((e = transport_occupancy_exact(smem, &per_sm)) != cudaSuccess || per_sm < 1)
            return reject(LP_ERR_CUDA, "lp_run_noalloc: occupancy query failed");
        if ((e = launch_transport_exact(P, sms * per_sm, smem, s)) != cudaSuccess)
            return reject(LP_ERR_CUDA, "lp_run_noalloc: transport launch failed");
    }
    if (a->counters) {
        e = cudaMemcpyAsync(a->counters, sb + OFF_CNT, LP_NCOUNTERS * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s);
        if (e != cudaSuccess) return reject(LP_ERR_CUDA, "lp_run_noalloc: counter copy failed");
    }
    return LP_OK;
}
