// lp_batch_impl.cuh -- one persistent launch over many transport instances.
//
// An instance is one complete transport problem: a mesh (BVH + cell grid), a table of
// optical properties, a photon budget and its own tallies, described by a KParams in
// device memory.  The reference runs one such problem per program run
// (CalculatePropagation::ExecKernel, CalculatePropagation.cpp:1389-1759); here a whole
// set of them -- meshes x wavelengths x optical-property draws with uneven budgets --
// runs in one launch, so the GPU drains once instead of once per problem.
//
// Work distribution: each warp is bound to one instance at a time and keeps a copy of
// its KParams, mesh view and media table in its own shared-memory slot.  Lanes whose
// photon ended take new photon indices of that instance with one atomicAdd per warp
// refill on the instance's claim counter.  When the instance has no unclaimed photons
// left, the warp finishes the photons it holds, adds its counters to the instance's,
// and binds the next instance with unclaimed photons (a shared frontier index moves
// past exhausted instances).  A photon is traced by exactly the same device functions
// as in transport_kernel, with the same Philox counter (photon id, event, stream), so
// an instance's integer tallies equal those of a single-instance run bit for bit.
#pragma once
#include "lp_transport_impl.cuh"

namespace lp {

struct WarpSlot {
    KParams P;
    MeshView M;
    Medium media[kBatchMedia];
};

__device__ __forceinline__ void warp_flush_counters(const KParams &P, const Counters &c, uint32_t photons,
                                                    unsigned lane)
{
    const uint32_t v[10] = {c.scatter, c.boundary, c.query, c.roulette, c.rz_drop, c.vox_drop, photons, c.skip,
                            c.bvh, 0u};
    const int slot[9] = {0, 1, 2, 3, 6, 7, 8, 10, 11};
#pragma unroll
    for (int i = 0; i < 9; ++i) {
        unsigned long long x = v[i];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0 && x) atomicAdd(P.counters + slot[i], x);
    }
}

// Copy instance `i` into the warp's slot (all 32 lanes take part).
__device__ __forceinline__ void warp_load_slot(WarpSlot &S, const KParams *inst, int i, unsigned lane)
{
    const uint32_t *src = reinterpret_cast<const uint32_t *>(inst + i);
    uint32_t *dst = reinterpret_cast<uint32_t *>(&S.P);
    for (unsigned k = lane; k < sizeof(KParams) / 4; k += 32) dst[k] = __ldg(src + k);
    __syncwarp();
    const uint32_t *ms = reinterpret_cast<const uint32_t *>(S.P.media);
    uint32_t *md = reinterpret_cast<uint32_t *>(S.media);
    const unsigned words = (unsigned)S.P.n_media * (sizeof(Medium) / 4);
    for (unsigned k = lane; k < words; k += 32) md[k] = __ldg(ms + k);
    if (lane == 0) {
        MeshView &M = S.M;
        M.na = S.P.node_a; M.nb = S.P.node_b; M.nc = S.P.node_c; M.nd = S.P.node_d;
        M.ta = S.P.tri_a; M.tb = S.P.tri_b; M.tc = S.P.tri_c;
        M.s_na = M.s_nb = M.s_nc = nullptr;
        M.s_nd = nullptr;
        M.s_ta = M.s_tb = M.s_tc = nullptr;
        M.nodes_smem = 0;
        M.tris_smem = 0;
        M.n_nodes = S.P.n_nodes;
        M.n_tri = S.P.n_tri;
        M.dbg = S.P.counters ? S.P.counters + kBoundsCounter : nullptr;
        M.tri_eps = S.P.tri_eps;
    }
    __syncwarp();
}

__device__ __forceinline__ void zero_grad(GradAcc &ga, int n_media)
{
    for (int r = 0; r < n_media; ++r) {
        ga.L[r] = 0.0f;
        ga.k[r] = 0;
    }
}

template <bool Exact, bool Grad, int BLOCK, int MINB, int STACK>
__global__ void __launch_bounds__(BLOCK, MINB) batch_kernel(const __grid_constant__ BatchParams B)
{
    __shared__ WarpSlot slots[BLOCK / 32];
    const unsigned lane = threadIdx.x & 31u;
    const unsigned lt_mask = (1u << lane) - 1u;
    WarpSlot &S = slots[threadIdx.x >> 5];
    Counters cnt = {};
    uint32_t photons = 0;
    Photon ph;
    GradAcc ga;
    bool alive = false;
    int inst = -1;
    bool exhausted = true;   // the bound instance has no unclaimed photons (or none is bound)
    for (;;) {
        const unsigned need = __ballot_sync(0xffffffffu, !alive);
        if (need == 0xffffffffu && exhausted) {
            // every lane is idle: close the instance, bind the next one with unclaimed photons
            if (inst >= 0) {
                warp_flush_counters(S.P, cnt, photons, lane);
                cnt = Counters{};
                photons = 0;
            }
            int next = -1;
            unsigned long long base = 0;
            if (lane == 0) {
                int f = atomicAdd(B.frontier, 0);
                for (; f < B.n_inst; ++f) {
                    const unsigned long long b = atomicAdd(B.claimed + f, 32ull);
                    if (b < (unsigned long long)B.inst[f].n) {
                        next = f;
                        base = b;
                        break;
                    }
                    atomicCAS(B.frontier, f, f + 1);
                }
            }
            next = __shfl_sync(0xffffffffu, next, 0);
            if (next < 0) break;
            base = __shfl_sync(0xffffffffu, base, 0);
            __syncwarp();
            warp_load_slot(S, B.inst, next, lane);
            inst = next;
            const unsigned long long n = (unsigned long long)S.P.n;
            exhausted = base + 32ull >= n;
            const unsigned long long idx = base + lane;
            if (idx < n) {
                start_photon(S.P, ph, (uint32_t)idx);
                if (Grad) zero_grad(ga, S.P.n_media);
                alive = true;
            }
        } else if (need && !exhausted) {
            const int k = __popc(need);
            unsigned long long base = 0;
            if (lane == 0) base = atomicAdd(B.claimed + inst, (unsigned long long)k);
            base = __shfl_sync(0xffffffffu, base, 0);
            const unsigned long long n = (unsigned long long)S.P.n;
            if (base + (unsigned long long)k >= n) exhausted = true;
            if (!alive) {
                const unsigned long long idx = base + __popc(need & lt_mask);
                if (idx < n) {
                    start_photon(S.P, ph, (uint32_t)idx);
                    if (Grad) zero_grad(ga, S.P.n_media);
                    alive = true;
                }
            }
        }
        if (alive) {
            if (!step_photon<Exact, Grad, STACK>(S.P, S.M, S.media, S.P.region, S.P.counters, ph, cnt, &ga)) {
                if (ph.region_acc) atomicAdd(S.P.region + ph.curr, ph.region_acc);
                if (Grad) {
                    ga.L[ph.curr] += ph.seg_len;
                    ga.k[ph.curr] += ph.seg_k;
                }
                finish_photon<Grad>(S.P, ph, Grad ? &ga : nullptr);
                photons++;
                alive = false;
            }
        }
    }
    if (inst >= 0) warp_flush_counters(S.P, cnt, photons, lane);
}

template <bool Exact, bool Grad, int BLOCK, int MINB, int STACK>
cudaError_t launch_batch_t(const BatchParams &B, int grid, cudaStream_t s)
{
    batch_kernel<Exact, Grad, BLOCK, MINB, STACK><<<grid, BLOCK, 0, s>>>(B);
    return cudaGetLastError();
}

template <bool Exact, bool Grad, int BLOCK, int MINB, int STACK>
cudaError_t batch_occupancy_t(int *blocks_per_sm)
{
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, batch_kernel<Exact, Grad, BLOCK, MINB, STACK>,
                                                         BLOCK, 0);
}

}  // namespace lp
