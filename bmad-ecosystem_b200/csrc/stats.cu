// stats.cu -- bunch statistics on the device for the long-term-tracking outputs.
//
// The sums ltt_calc_bunch_data (bsim/modules/lt_tracking_mod.f90:2369-2451) and
// calc_bunch_sigma_matrix_etc (bmad/multiparticle/beam_utils.f90:1757-1844) take over the live
// particles, in two passes as they do (the centred sums need the average first):
//   pass 1: count, sum vec_i, sum t, sum t^2, sum vec_i vec_j (i <= j)            (30 values)
//   pass 2: sum (vec_i - a_i)(vec_j - a_j) (i <= j), sum (vec_i - a_i)^3, ^4       (33 values)
// Each pass is a grid of kStatBlocks CTAs writing per-CTA partial sums (warp shuffles, then the
// warps in order) and one reduce kernel that adds the partials in CTA order, so the result does
// not depend on scheduling. The host turns the sums into the bunch data (bunchdata.cpp).

#include <cuda_runtime.h>

#include "stats.cuh"

namespace bmadgpu {

namespace {

constexpr int kStatThreads = 256;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Adds the block's NV values (one per thread-local accumulator) and writes them to out[NV].
template <int NV>
__device__ void block_sum(double (&acc)[NV], double* __restrict__ out) {
  __shared__ double part[kStatThreads / 32][NV];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < NV; k++) {
    double s = warp_sum(acc[k]);
    if (lane == 0) part[warp][k] = s;
  }
  __syncthreads();
  for (int k = threadIdx.x; k < NV; k += kStatThreads) {
    double s = 0;
    for (int w = 0; w < kStatThreads / 32; w++) s += part[w][k];
    out[k] = s;
  }
}

__global__ void __launch_bounds__(kStatThreads) k_stats_pass1(const double* __restrict__ vec,
                                                              const double* __restrict__ t,
                                                              const int32_t* __restrict__ state, int64_t n,
                                                              double* __restrict__ partial) {
  double acc[kStatPass1] = {0};
  for (int64_t j = (int64_t)blockIdx.x * kStatThreads + threadIdx.x; j < n; j += (int64_t)gridDim.x * kStatThreads) {
    if (state[j] != 1) continue;
    double v[6];
#pragma unroll
    for (int i = 0; i < 6; i++) v[i] = vec[i * n + j];
    const double tj = t ? t[j] : 0.0;
    acc[0] += 1;
#pragma unroll
    for (int i = 0; i < 6; i++) acc[1 + i] += v[i];
    acc[7] += tj;
    acc[8] += tj * tj;
    int k = 9;
#pragma unroll
    for (int i = 0; i < 6; i++)
#pragma unroll
      for (int m = i; m < 6; m++) acc[k++] += v[i] * v[m];
  }
  block_sum<kStatPass1>(acc, partial + (int64_t)blockIdx.x * kStatPass1);
}

__global__ void __launch_bounds__(kStatThreads) k_stats_pass2(const double* __restrict__ vec,
                                                              const int32_t* __restrict__ state, int64_t n,
                                                              const double* __restrict__ sums1,
                                                              double* __restrict__ partial) {
  double acc[kStatPass2] = {0};
  const double cnt = sums1[0];
  double a[6];
#pragma unroll
  for (int i = 0; i < 6; i++) a[i] = cnt > 0 ? sums1[1 + i] / cnt : 0.0;
  for (int64_t j = (int64_t)blockIdx.x * kStatThreads + threadIdx.x; j < n; j += (int64_t)gridDim.x * kStatThreads) {
    if (state[j] != 1) continue;
    double d[6];
#pragma unroll
    for (int i = 0; i < 6; i++) d[i] = vec[i * n + j] - a[i];
    int k = 0;
#pragma unroll
    for (int i = 0; i < 6; i++)
#pragma unroll
      for (int m = i; m < 6; m++) acc[k++] += d[i] * d[m];
#pragma unroll
    for (int i = 0; i < 6; i++) {
      const double d2 = d[i] * d[i];
      acc[21 + i] += d2 * d[i];
      acc[27 + i] += d2 * d2;
    }
  }
  block_sum<kStatPass2>(acc, partial + (int64_t)blockIdx.x * kStatPass2);
}

// out[k] = sum over CTAs, in CTA order, of partial[cta][k].
__global__ void k_stats_reduce(const double* __restrict__ partial, int nv, int n_blocks, double* __restrict__ out) {
  for (int k = threadIdx.x; k < nv; k += blockDim.x) {
    double s = 0;
    for (int b = 0; b < n_blocks; b++) s += partial[(int64_t)b * nv + k];
    out[k] = s;
  }
}

}  // namespace

cudaError_t launch_bunch_sums(const double* vec, const double* t, const int32_t* state, int64_t n, double* partial,
                              double* sums, cudaStream_t stream) {
  k_stats_pass1<<<kStatBlocks, kStatThreads, 0, stream>>>(vec, t, state, n, partial);
  k_stats_reduce<<<1, 64, 0, stream>>>(partial, kStatPass1, kStatBlocks, sums);
  k_stats_pass2<<<kStatBlocks, kStatThreads, 0, stream>>>(vec, state, n, sums, partial);
  k_stats_reduce<<<1, 64, 0, stream>>>(partial, kStatPass2, kStatBlocks, sums + kStatPass1);
  return cudaGetLastError();
}

}  // namespace bmadgpu
