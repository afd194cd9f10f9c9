// stats.cuh -- device sums for the bunch statistics (stats.cu) and their host reduction
// (bunchdata.cpp).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace bmadgpu {

constexpr int kStatBlocks = 296;   // fixed CTA count: the reduction order does not depend on the GPU
constexpr int kStatPass1 = 30;     // count, sum v (6), sum t, sum t^2, sum v_i v_j (21)
constexpr int kStatPass2 = 33;     // centred sum d_i d_j (21), sum d^3 (6), sum d^4 (6)
constexpr int kStatSums = kStatPass1 + kStatPass2;

// partial: kStatBlocks * kStatPass2 doubles of scratch; sums: kStatSums doubles (device).
cudaError_t launch_bunch_sums(const double* vec, const double* t, const int32_t* state, int64_t n, double* partial,
                              double* sums, cudaStream_t stream);

}  // namespace bmadgpu
