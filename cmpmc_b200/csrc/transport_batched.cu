// transport_batched.cu -- the batched FP32 form (per-primary substreams).
#include "device.cuh"

namespace cmpmc_gpu {

cudaError_t launch_batched_fp32(const Lattice&, const Detector&, const RunArgs&, int, int, cudaStream_t) {
    return cudaErrorNotSupported;
}

cudaError_t batched_fp32_occupancy(int, int* blocks_per_sm) {
    *blocks_per_sm = 1;
    return cudaSuccess;
}

}  // namespace cmpmc_gpu
