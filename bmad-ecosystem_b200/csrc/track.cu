// track.cu -- sm_100a kernels for multi-turn bunch tracking.
//
// k_track: one thread per particle; the particle lives in registers for all n_turns turns of
// the launch, running the element loop of track_bunch (bmad/multiparticle/beam_mod.f90:159-166)
// with the per-element wrapper of track1 (bmad/code/track1.f90:179-329) around each map. The
// packed element table is staged once per CTA into shared memory by a TMA bulk copy
// (cp.async.bulk, mbarrier completion, bounded wait), so the element loop reads invariants with
// broadcast shared-memory loads. Lost particles leave the loop at once and record where they
// were lost (state, element, turn, location) as track1_bunch_hom leaves them
// (bmad/multiparticle/beam_utils.f90:81-86). Optional per-turn sums over live particles
// (n_live, <x_i>, <x_i x_j>; bsim/modules/lt_tracking_mod.f90:2393-2421) are reduced with warp
// shuffles and one atomic per warp and value.
//
// k_compact: warp ballot / popc stream compaction of the live-particle index list.

// The plain tracking kernel takes quotients with a common divisor from one rounded reciprocal
// (maps.cuh, div_rcp): the same bits as the division, measured faster in this kernel.
#define BG_SHARED_RECIPROCAL
#include <cuda_runtime.h>

#include "particle.cuh"
#include "tma.cuh"
#include "track.cuh"
#include "batch.cuh"

namespace bmadgpu {
cudaError_t adjoint_upload_constants();  // adjoint.cu
}

namespace bmadgpu {

namespace {

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ void add_moments(const Particle& p, bool alive, double* __restrict__ m) {
  const double v[6] = {p.x, p.px, p.y, p.py, p.z, p.pz};
  const int lane = threadIdx.x & 31;
  double s = warp_sum(alive ? 1.0 : 0.0);
  if (lane == 0 && s != 0) atomicAdd(m, s);
  if (__any_sync(0xffffffffu, alive) == 0) return;
  int k = 7;
#pragma unroll
  for (int i = 0; i < 6; i++) {
    double si = warp_sum(alive ? v[i] : 0.0);
    if (lane == 0) atomicAdd(m + 1 + i, si);
#pragma unroll
    for (int j = i; j < 6; j++) {
      double sij = warp_sum(alive ? v[i] * v[j] : 0.0);
      if (lane == 0) atomicAdd(m + k, sij);
      k++;
    }
  }
}

template <int BLOCK, int MINB, bool FULL>
__global__ void __launch_bounds__(BLOCK, MINB) k_track(const TrackArgs a, int stage_smem) {
  extern __shared__ __align__(128) uint8_t smem[];
  __shared__ __align__(8) uint64_t bar;
  const uint8_t* tbl = a.table;
  bool staged = false;
  if (stage_smem) {
    if (threadIdx.x == 0) mbar_init(&bar, 1);
    __syncthreads();
    if (threadIdx.x == 0) {
      stage_table_issue(smem, a.table, a.table_bytes, &bar);
    }
    const bool ok = mbar_wait_bounded(&bar, 0);
    // Every thread must agree; a timed-out copy falls back to reading the table from global
    // memory and raises the error flag for the host.
    staged = __syncthreads_and(ok);
    if (!staged && threadIdx.x == 0) atomicOr(a.err_flag, 1);
    if (staged) tbl = smem;
  }
  const EleHdr* hdr = reinterpret_cast<const EleHdr*>(tbl);
  const ApRec* ap = reinterpret_cast<const ApRec*>(tbl + a.hdr_bytes);
  const double* pool = reinterpret_cast<const double*>(tbl + a.hdr_bytes + a.ap_bytes);
  const Globals G = a.G;
  const int64_t n_work = *a.n_work;
  const double seg_ref = a.ref_prefix[a.ix_end] - a.ref_prefix[a.ix_start];

  const SoA soa{a.vec, a.beta, a.t, a.state, a.ix_ele, a.ix_turn, a.location, a.ld};

  for (int64_t base = (int64_t)blockIdx.x * BLOCK; base < n_work; base += (int64_t)gridDim.x * BLOCK) {
    const int64_t w = base + threadIdx.x;
    const bool valid = w < n_work;
    const int64_t j = valid ? (a.live ? (int64_t)a.live[w] : w) : 0;
    Particle p;
    p.state = 0;
    if (valid) load_particle(soa, j, p);
    bool alive = valid && p.state == S_ALIVE;
    const double z_in = p.z, beta_in = p.beta;
    LossInfo li;
    if (alive) refresh(p, G);
    for (int turn = 0; turn < a.n_turns; ++turn) {
      if (alive) alive = track_turn<FULL>(p, hdr, pool, ap, G, a.ix_start, a.ix_end, turn == 0, a.turn0 + turn, li);
      if (a.moments) add_moments(p, alive, a.moments + (int64_t)turn * 28);
    }
    if (valid) store_particle(soa, j, p, alive, li, z_in, beta_in, a.n_turns, a.turn0, seg_ref, a.ref_prefix, a.ix_start);
  }
  if (stage_smem && !staged) {
    // Let our own bulk copy drain (bounded) before the CTA's shared memory is released.
    mbar_wait_bounded(&bar, 0);
  }
}

__global__ void k_compact(const int32_t* __restrict__ state, const int32_t* __restrict__ live_in,
                          const int64_t* __restrict__ n_in, int32_t* __restrict__ live_out,
                          unsigned long long* __restrict__ n_out) {
  const int64_t n = *n_in;
  const int lane = threadIdx.x & 31;
  for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < n; base += (int64_t)gridDim.x * blockDim.x) {
    int64_t w = base + threadIdx.x;
    int32_t j = (w < n) ? (live_in ? live_in[w] : (int32_t)w) : 0;
    bool keep = (w < n) && state[j] == S_ALIVE;
    unsigned mask = __ballot_sync(0xffffffffu, keep);
    unsigned long long off = 0;
    if (lane == 0 && mask) off = atomicAdd(n_out, (unsigned long long)__popc(mask));
    off = __shfl_sync(0xffffffffu, off, 0);
    if (keep) live_out[off + __popc(mask & ((1u << lane) - 1))] = j;
  }
}

// FP64 peak probe: 8 independent DFMA chains per thread, register resident.
__global__ void k_fp64_peak(double* out, int iters, double a, double b) {
  double r[8];
#pragma unroll
  for (int k = 0; k < 8; k++) r[k] = threadIdx.x * 1e-9 + k;
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int k = 0; k < 8; k++) r[k] = fma(r[k], a, b);
  }
  double s = 0;
#pragma unroll
  for (int k = 0; k < 8; k++) s += r[k];
  if (s == 123.456) out[0] = s;  // keeps the chains live
}

}  // namespace

cudaError_t measure_fp64_peak(int sm_count, cudaStream_t stream, double* flops_per_s) {
  double* d = nullptr;
  cudaError_t e = cudaMalloc(&d, sizeof(double));
  if (e != cudaSuccess) return e;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int block = 256, iters = 1 << 14;
  const int grid = sm_count * 8;
  k_fp64_peak<<<grid, block, 0, stream>>>(d, 64, 0.999999, 1e-7);  // warm-up
  cudaEventRecord(e0, stream);
  k_fp64_peak<<<grid, block, 0, stream>>>(d, iters, 0.999999, 1e-7);
  cudaEventRecord(e1, stream);
  e = cudaEventSynchronize(e1);
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(d);
  if (e != cudaSuccess) return e;
  double flops = 2.0 * 8 * (double)iters * block * (double)grid;
  *flops_per_s = flops / (ms * 1e-3);
  return cudaGetLastError();
}

int table_fits_smem(uint32_t table_bytes) { return table_bytes <= 200 * 1024; }

cudaError_t upload_constants() {
  // the __constant__ tables exist once per translation unit: fill this one's and the batch kernel's
  double cm[22][22], cf[22][22];
  build_cmulti_tables(cm, cf);
  cudaError_t e = cudaMemcpyToSymbol(c_cmulti, cm, sizeof(cm));
  if (e != cudaSuccess) return e;
  e = cudaMemcpyToSymbol(c_cfull, cf, sizeof(cf));
  if (e != cudaSuccess) return e;
  e = batch_upload_constants();
  if (e != cudaSuccess) return e;
  e = batch_rec_upload_constants();
  if (e != cudaSuccess) return e;
  return adjoint_upload_constants();
}

// Kernel variants: threads per CTA x minimum resident CTAs per SM (the register budget per
// thread follows: 65536 / (BLOCK * MINB), capped at 255).
struct Variant {
  int block, minb;
  const void* fn;       // the kernel for every element form
  const void* fn_lean;  // the kernel for tables without rare forms (TableInfo::rare = 0)
};
#define BG_VARIANT(B, M) {B, M, (const void*)k_track<B, M, true>, (const void*)k_track<B, M, false>}
static const Variant kVariants[] = {
    BG_VARIANT(64, 8),   BG_VARIANT(64, 12), BG_VARIANT(128, 3), BG_VARIANT(128, 4), BG_VARIANT(128, 5),
    BG_VARIANT(128, 6),  BG_VARIANT(256, 2), BG_VARIANT(256, 1), BG_VARIANT(256, 3), BG_VARIANT(512, 1),
};
#undef BG_VARIANT

cudaError_t launch_track(const TrackArgs& a, const LaunchCfg& cfg, int sm_count, cudaStream_t stream) {
  int stage = (cfg.stage_smem && table_fits_smem(a.table_bytes)) ? 1 : 0;
  // ctas_per_sm selects the register budget: the variant with the largest minimum CTA count
  // not above it (0: the most registers per thread)
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
  if (!v) return cudaErrorInvalidValue;
  const void* fn = a.rare ? v->fn : v->fn_lean;
  int per_sm = 0;
  cudaError_t err;
  if (stage) {
    // Staging is taken only where it costs no residency: a table whose copy would leave room
    // for fewer CTAs per SM than the registers allow (the multipole pool of a large ring can
    // take most of the shared memory) is read through L1 instead, which measured ~2.8x faster
    // on a 176 KB table than one staged CTA per SM.
    int plain_sm = 0;
    if ((err = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, 0)) != cudaSuccess) return err;
    if ((err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&plain_sm, fn, cfg.block, 0)) != cudaSuccess) return err;
    if ((err = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)a.table_bytes)) !=
        cudaSuccess)
      return err;
    if ((err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, cfg.block, a.table_bytes)) != cudaSuccess)
      return err;
    if (per_sm < plain_sm) stage = 0;
  }
  const size_t smem = stage ? a.table_bytes : 0;
  err = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (err != cudaSuccess) return err;
  err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, cfg.block, smem);
  if (err != cudaSuccess) return err;
  if (per_sm < 1) per_sm = 1;
  // Persistent grid: one full wave; every CTA strides over the particle range.
  int64_t grid = (int64_t)sm_count * per_sm;
  void* args[] = {(void*)&a, (void*)&stage};
  return cudaLaunchKernel(fn, dim3((unsigned)grid), dim3(cfg.block), args, smem, stream);
}

cudaError_t launch_compact(const int32_t* state, const int32_t* live_in, const int64_t* n_in, int64_t n_max,
                           int32_t* live_out, int64_t* n_out, cudaStream_t stream) {
  cudaError_t err = cudaMemsetAsync(n_out, 0, sizeof(int64_t), stream);
  if (err != cudaSuccess) return err;
  int64_t blocks = (n_max + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  if (blocks < 1) blocks = 1;
  k_compact<<<(unsigned)blocks, 256, 0, stream>>>(state, live_in, n_in, live_out,
                                                   reinterpret_cast<unsigned long long*>(n_out));
  return cudaGetLastError();
}

}  // namespace bmadgpu
