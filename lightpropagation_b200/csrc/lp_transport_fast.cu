// lp_transport_fast.cu -- production instantiation of the transport kernel
// (Exact = false; every unit is built with --fmad=false, the production arithmetic
// writes its fused multiply-adds explicitly; see lp_transport_impl.cuh).
#include "lp_transport_impl.cuh"

namespace lp {

cudaError_t launch_transport_fast(const KParams &P, int grid, int smem, cudaStream_t s)
{
    return launch_transport_t<false>(P, grid, smem, s);
}

cudaError_t transport_occupancy_fast(int smem, int *blocks_per_sm)
{
    return transport_occupancy_t<false, false>(smem, blocks_per_sm);
}

cudaError_t transport_occupancy_fast_grad(int smem, int *blocks_per_sm)
{
    return transport_occupancy_t<false, true>(smem, blocks_per_sm);
}

}  // namespace lp
