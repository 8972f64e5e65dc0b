// lp_transport_batch.cu -- instantiations of the batched transport kernel
// (production arithmetic) for the launch configurations the autotuner chooses from.
#include "lp_batch_impl.cuh"

namespace lp {

// (threads per block, minimum resident blocks per SM for the register budget,
//  BVH traversal stack entries)
struct BatchConfig {
    int block, min_blocks, stack;
};
static const BatchConfig kBatchConfigs[] = {{256, 3, 64}, {128, 6, 64}, {256, 2, 64}, {256, 3, 32}, {512, 1, 64}};
constexpr int kNumBatchConfigs = 5;

int batch_config_count() { return kNumBatchConfigs; }

int batch_config_info(int config, int *block, int *min_blocks, int *stack)
{
    if (config < 0 || config >= kNumBatchConfigs) return 1;
    *block = kBatchConfigs[config].block;
    *min_blocks = kBatchConfigs[config].min_blocks;
    *stack = kBatchConfigs[config].stack;
    return 0;
}

template <bool Grad>
static cudaError_t launch_cfg(int config, const BatchParams &B, int grid, cudaStream_t s)
{
    switch (config) {
    case 0: return launch_batch_t<false, Grad, 256, 3, 64>(B, grid, s);
    case 1: return launch_batch_t<false, Grad, 128, 6, 64>(B, grid, s);
    case 2: return launch_batch_t<false, Grad, 256, 2, 64>(B, grid, s);
    case 3: return launch_batch_t<false, Grad, 256, 3, 32>(B, grid, s);
    case 4: return launch_batch_t<false, Grad, 512, 1, 64>(B, grid, s);
    default: return cudaErrorInvalidValue;
    }
}

template <bool Grad>
static cudaError_t occupancy_cfg(int config, int *per_sm)
{
    switch (config) {
    case 0: return batch_occupancy_t<false, Grad, 256, 3, 64>(per_sm);
    case 1: return batch_occupancy_t<false, Grad, 128, 6, 64>(per_sm);
    case 2: return batch_occupancy_t<false, Grad, 256, 2, 64>(per_sm);
    case 3: return batch_occupancy_t<false, Grad, 256, 3, 32>(per_sm);
    case 4: return batch_occupancy_t<false, Grad, 512, 1, 64>(per_sm);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_batch(int config, bool grad, const BatchParams &B, int grid, cudaStream_t s)
{
    return grad ? launch_cfg<true>(config, B, grid, s) : launch_cfg<false>(config, B, grid, s);
}

cudaError_t batch_occupancy(int config, bool grad, int *blocks_per_sm)
{
    return grad ? occupancy_cfg<true>(config, blocks_per_sm) : occupancy_cfg<false>(config, blocks_per_sm);
}

}  // namespace lp
