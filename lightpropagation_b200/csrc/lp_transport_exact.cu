// lp_transport_exact.cu -- reference-arithmetic instantiation of the transport kernel
// (Exact = true, compiled with --fmad=false), the BVH query kernel used to verify the
// traversal against the brute-force scan, and small utility kernels.
#include "lp_transport_impl.cuh"

namespace lp {

cudaError_t launch_transport_exact(const KParams &P, int grid, int smem, cudaStream_t s)
{
    return launch_transport_t<true>(P, grid, smem, s);
}

cudaError_t transport_occupancy_exact(int smem, int *blocks_per_sm)
{
    return transport_occupancy_t<true, false>(smem, blocks_per_sm);
}

cudaError_t transport_occupancy_exact_grad(int smem, int *blocks_per_sm)
{
    return transport_occupancy_t<true, true>(smem, blocks_per_sm);
}

__global__ void __launch_bounds__(kBlock) query_kernel(const __grid_constant__ KParams P, int64_t n,
                                                       const float *orig, const float *dir,
                                                       const int32_t *ref, const float *tmax,
                                                       int32_t *id_out, float *t_out)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const SmemLayout L = smem_layout(P.nodes_smem, P.tris_smem);
    const MeshView M = stage_mesh(P, smem, L);
    __syncthreads();
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const V3 p = v3(orig[3 * i], orig[3 * i + 1], orig[3 * i + 2]);
        const V3 v = v3(dir[3 * i], dir[3 * i + 1], dir[3 * i + 2]);
        float t;
        bool used_bvh;
        id_out[i] = cell_query(P, M, p, v, ref[i], tmax[i], t, used_bvh);
        t_out[i] = t;
    }
}

__global__ void philox_kernel(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0,
                              uint32_t k1, int64_t n, uint32_t *out)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        uint32_t a = c0, b = c1, c = c2 + (uint32_t)i, d = c3;
        philox4x32_10(a, b, c, d, k0, k1);
        out[4 * i] = a; out[4 * i + 1] = b; out[4 * i + 2] = c; out[4 * i + 3] = d;
    }
}

// FP32 throughput probe: 8 independent FMA chains per thread.  2 flops per FMA.
__global__ void __launch_bounds__(256) fma_peak_kernel(float *out, int iters, float a, float b)
{
    float x0 = threadIdx.x * 1e-3f, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3;
    float x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6, x7 = x0 + 7;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            x0 = __fmaf_rn(x0, a, b); x1 = __fmaf_rn(x1, a, b); x2 = __fmaf_rn(x2, a, b); x3 = __fmaf_rn(x3, a, b);
            x4 = __fmaf_rn(x4, a, b); x5 = __fmaf_rn(x5, a, b); x6 = __fmaf_rn(x6, a, b); x7 = __fmaf_rn(x7, a, b);
        }
    }
    const float s = ((x0 + x1) + (x2 + x3)) + ((x4 + x5) + (x6 + x7));
    if (s == 1234.5f) out[0] = s;  // keeps the chains alive; practically never taken
}

// 64-bit atomic adds whose results are not used (reductions at the L2), each lane of a
// warp to its own pseudo-random slot of an L2-resident buffer: the access pattern of the
// transport kernel's absorption deposits.
__global__ void __launch_bounds__(256) red_peak_kernel(unsigned long long *buf, uint32_t mask, int iters)
{
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t h = g * 0x9E3779B1u + 0x7F4A7C15u;
    for (int i = 0; i < iters; ++i) {
        h ^= h >> 15;
        h *= 0x2C1B3C6Du;
        h ^= h >> 12;
        atomicAdd(buf + (h & mask), 1ull);
    }
}

int smem_bytes(int nodes_smem, int tris_smem) { return smem_layout(nodes_smem, tris_smem).bytes; }

int block_size() { return kBlock; }

cudaError_t launch_query(const KParams &P, int smem, int64_t n, const float *orig, const float *dir,
                         const int32_t *ref, const float *tmax, int32_t *id_out, float *t_out,
                         cudaStream_t s)
{
    cudaError_t e = cudaFuncSetAttribute(query_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    int grid = (int)std::min<int64_t>((n + kBlock - 1) / kBlock, 148 * 8);
    if (grid < 1) grid = 1;
    query_kernel<<<grid, kBlock, smem, s>>>(P, n, orig, dir, ref, tmax, id_out, t_out);
    return cudaGetLastError();
}

cudaError_t launch_philox(const uint32_t *ctr, const uint32_t *key, int64_t n, uint32_t *out, cudaStream_t s)
{
    int grid = (int)std::min<int64_t>((n + 255) / 256, 148 * 8);
    if (grid < 1) grid = 1;
    philox_kernel<<<grid, 256, 0, s>>>(ctr[0], ctr[1], ctr[2], ctr[3], key[0], key[1], n, out);
    return cudaGetLastError();
}

double fma_peak_tflops(int num_sms)
{
    float *d = nullptr;
    if (cudaMalloc(&d, 16) != cudaSuccess) return 0.0;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int blocks = num_sms * 8, threads = 256, iters = 4096;
    fma_peak_kernel<<<blocks, threads>>>(d, 64, 0.999f, 1e-3f);  // warm-up
    double best = 0.0;
    for (int r = 0; r < 3; ++r) {
        cudaEventRecord(e0);
        fma_peak_kernel<<<blocks, threads>>>(d, iters, 0.999f, 1e-3f);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        const double flops = 2.0 * 8 * 16 * (double)iters * blocks * threads;
        if (ms > 0) best = std::max(best, flops / (ms * 1e-3) / 1e12);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(d);
    return best;
}

// Throughput of 64-bit atomic reductions to an L2-resident buffer (16 MB), in atomics/s.
double red_peak_per_s(int num_sms)
{
    const uint32_t slots = 1u << 21;   // 16 MB of uint64
    unsigned long long *d = nullptr;
    if (cudaMalloc(&d, (size_t)slots * 8) != cudaSuccess) return 0.0;
    cudaMemset(d, 0, (size_t)slots * 8);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int blocks = num_sms * 8, threads = 256, iters = 512;
    red_peak_kernel<<<blocks, threads>>>(d, slots - 1, 16);   // warm-up
    double best = 0.0;
    for (int r = 0; r < 3; ++r) {
        cudaEventRecord(e0);
        red_peak_kernel<<<blocks, threads>>>(d, slots - 1, iters);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        const double n = (double)iters * blocks * threads;
        if (ms > 0) best = std::max(best, n / (ms * 1e-3));
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(d);
    return best;
}

}  // namespace lp
