// batch.cu -- batched tracking of many lattice variants in one persistent launch.
//
// k_batch_track: a persistent grid (one full wave of CTAs) pulls work items from a device
// counter. An item is (variant, tile of `tile` consecutive entries of the variant's live list);
// items of variant v are numbered tile_prefix[v] .. tile_prefix[v+1]-1. A CTA that moves to a
// new variant re-stages that variant's element table into shared memory with a bulk copy
// (mbarrier completion, bounded wait, the phase bit flipping on every use). Each thread tracks
// `ppt` particles of the tile one after another, each through all turns of the launch, with the
// same per-particle code as k_track (particle.cuh). Survivors are appended to the variant's next
// live list with a warp ballot and one atomic per warp, so compaction needs no extra pass.
//
// k_batch_plan: one CTA; exclusive scan of the tile counts (live count / tile, rounded up) over
// the variants, reset of the work counter and of the next launch's live counts.

#include <cuda_runtime.h>

#include "batch.cuh"
#include "batch_kernel.cuh"
#include "particle.cuh"
#include "tma.cuh"
#include "track.cuh"

namespace bmadgpu {

namespace {

__global__ void k_batch_plan(const BatchVar* __restrict__ vars, int n_var, int tile, int turn_off, int identity,
                             const unsigned long long* __restrict__ n_in, int64_t* __restrict__ tile_prefix,
                             unsigned long long* __restrict__ queue, unsigned long long* __restrict__ n_zero) {
  __shared__ long long warp_sums[32];
  __shared__ long long carry;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, n_warps = blockDim.x >> 5;
  if (threadIdx.x == 0) {
    carry = 0;
    *queue = 0;
  }
  __syncthreads();
  for (int base = 0; base < n_var; base += blockDim.x) {
    const int v = base + threadIdx.x;
    long long tiles = 0;
    if (v < n_var) {
      const long long cnt = identity ? (long long)vars[v].n : (long long)n_in[v];
      if (vars[v].n_turns > turn_off && cnt > 0) tiles = (cnt + tile - 1) / tile;
      if (n_zero) n_zero[v] = 0;
    }
    long long x = tiles;  // inclusive scan within the warp
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const long long y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
      long long s = lane < n_warps ? warp_sums[lane] : 0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const long long y = __shfl_up_sync(0xffffffffu, s, o);
        if (lane >= o) s += y;
      }
      warp_sums[lane] = s;
    }
    __syncthreads();
    const long long excl = carry + (warp > 0 ? warp_sums[warp - 1] : 0) + x - tiles;
    if (v < n_var) tile_prefix[v] = excl;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry = excl + tiles;
    __syncthreads();
  }
  if (threadIdx.x == 0) tile_prefix[n_var] = carry;
}

__global__ void k_batch_set_turns(BatchVar* vars, int n_var, int turn0, int n_turns) {
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n_var; v += gridDim.x * blockDim.x) {
    vars[v].turn0 = turn0;
    vars[v].n_turns = n_turns;
  }
}

__global__ void k_batch_init_list(int32_t* __restrict__ list, int64_t n, unsigned long long* __restrict__ count) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    list[i] = (int32_t)i;
  if (blockIdx.x == 0 && threadIdx.x == 0) *count = (unsigned long long)n;
}

struct Variant {
  int block, minb;
  const void* fn;
  const void* fn_lean;
};
#define BG_BATCH_VARIANT(B, M) \
  {B, M, (const void*)k_batch_track<B, M, false, true>, (const void*)k_batch_track<B, M, false, false>}
const Variant kVariants[] = {
    BG_BATCH_VARIANT(64, 8),  BG_BATCH_VARIANT(64, 12), BG_BATCH_VARIANT(128, 3), BG_BATCH_VARIANT(128, 4),
    BG_BATCH_VARIANT(128, 5), BG_BATCH_VARIANT(128, 6), BG_BATCH_VARIANT(256, 1), BG_BATCH_VARIANT(256, 2),
    BG_BATCH_VARIANT(256, 3), BG_BATCH_VARIANT(512, 1),
};
#undef BG_BATCH_VARIANT

}  // namespace

// The multipole coefficient tables are __constant__ arrays of each translation unit; this one
// fills the copy the batch kernel reads.
cudaError_t batch_upload_constants() {
  double cm[22][22], cf[22][22];
  build_cmulti_tables(cm, cf);
  cudaError_t e = cudaMemcpyToSymbol(c_cmulti, cm, sizeof(cm));
  if (e != cudaSuccess) return e;
  return cudaMemcpyToSymbol(c_cfull, cf, sizeof(cf));
}

cudaError_t batch_resolve(const BatchLaunch& cfg, uint32_t smem_bytes, int sm_count, BatchKernel* out) {
  // same register-budget selection as launch_track
  const Variant* v = nullptr;
  for (const Variant& k : kVariants) {
    if (k.block != cfg.block) continue;
    if (cfg.ctas_per_sm > 0 && k.minb > cfg.ctas_per_sm) continue;
    if (!v || (cfg.ctas_per_sm > 0 ? k.minb > v->minb : k.minb < v->minb)) v = &k;
  }
  // no variant compiled for so few CTAs per SM: the one with the most registers per thread
  if (!v)
    for (const Variant& k : kVariants)
      if (k.block == cfg.block && (!v || k.minb < v->minb)) v = &k;
  if (!v || cfg.particles_per_thread < 1) return cudaErrorInvalidValue;
  cudaError_t err = cudaFuncSetAttribute(v->fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes);
  if (err != cudaSuccess) return err;
  const void* fn_rec = batch_rec_kernel(v->block, v->minb);
  if (!fn_rec) return cudaErrorInvalidValue;
  err = cudaFuncSetAttribute(fn_rec, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes);
  if (err != cudaSuccess) return err;
  int per_sm = 0;
  err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, v->fn, cfg.block, smem_bytes);
  if (err != cudaSuccess) return err;
  if (per_sm < 1) per_sm = 1;
  int per_sm_rec = 0;
  err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_rec, fn_rec, cfg.block, smem_bytes);
  if (err != cudaSuccess) return err;
  if (per_sm_rec < 1) per_sm_rec = 1;
  err = cudaFuncSetAttribute(v->fn_lean, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes);
  if (err != cudaSuccess) return err;
  int per_sm_lean = 0;
  err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_lean, v->fn_lean, cfg.block, smem_bytes);
  if (err != cudaSuccess) return err;
  if (per_sm_lean < 1) per_sm_lean = 1;
  out->fn_lean = v->fn_lean;
  out->grid_lean = sm_count * per_sm_lean;
  const void* fn_rec_lean = batch_rec_kernel(v->block, v->minb, false);
  if (!fn_rec_lean) return cudaErrorInvalidValue;
  err = cudaFuncSetAttribute(fn_rec_lean, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes);
  if (err != cudaSuccess) return err;
  int per_sm_rec_lean = 0;
  err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_rec_lean, fn_rec_lean, cfg.block, smem_bytes);
  if (err != cudaSuccess) return err;
  if (per_sm_rec_lean < 1) per_sm_rec_lean = 1;
  out->fn_rec_lean = fn_rec_lean;
  out->grid_rec_lean = sm_count * per_sm_rec_lean;
  out->fn = v->fn;
  out->fn_rec = fn_rec;
  out->grid_rec = sm_count * per_sm_rec;
  out->block = cfg.block;
  out->grid = sm_count * per_sm;
  out->ppt = cfg.particles_per_thread;
  out->smem = smem_bytes;
  return cudaSuccess;
}

cudaError_t batch_launch_track(const BatchKernel& k, const BatchArgs& a, cudaStream_t stream, bool record) {
  int ppt = k.ppt;
  void* args[] = {(void*)&a, (void*)&ppt};
  if (record && !a.rare)
    return cudaLaunchKernel(k.fn_rec_lean, dim3((unsigned)k.grid_rec_lean), dim3((unsigned)k.block), args, k.smem,
                            stream);
  if (record)
    return cudaLaunchKernel(k.fn_rec, dim3((unsigned)k.grid_rec), dim3((unsigned)k.block), args, k.smem, stream);
  if (!a.rare)
    return cudaLaunchKernel(k.fn_lean, dim3((unsigned)k.grid_lean), dim3((unsigned)k.block), args, k.smem, stream);
  return cudaLaunchKernel(k.fn, dim3((unsigned)k.grid), dim3((unsigned)k.block), args, k.smem, stream);
}

cudaError_t batch_launch_plan(const BatchVar* vars, int32_t n_var, int32_t tile, int32_t turn_off, bool identity,
                              const unsigned long long* n_in, int64_t* tile_prefix, unsigned long long* queue,
                              unsigned long long* n_zero, cudaStream_t stream) {
  k_batch_plan<<<1, 1024, 0, stream>>>(vars, n_var, tile, turn_off, identity ? 1 : 0, n_in, tile_prefix, queue,
                                       n_zero);
  return cudaGetLastError();
}

cudaError_t batch_launch_set_turns(BatchVar* vars, int32_t n_var, int32_t turn0, int32_t n_turns,
                                   cudaStream_t stream) {
  int blocks = (n_var + 255) / 256;
  if (blocks < 1) blocks = 1;
  if (blocks > 1024) blocks = 1024;
  k_batch_set_turns<<<blocks, 256, 0, stream>>>(vars, n_var, turn0, n_turns);
  return cudaGetLastError();
}

cudaError_t batch_launch_init_list(int32_t* list, int64_t n, unsigned long long* count, cudaStream_t stream) {
  int64_t blocks = (n + 255) / 256;
  if (blocks < 1) blocks = 1;
  if (blocks > 1024) blocks = 1024;
  k_batch_init_list<<<(unsigned)blocks, 256, 0, stream>>>(list, n, count);
  return cudaGetLastError();
}

}  // namespace bmadgpu
