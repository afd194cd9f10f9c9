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
#include "particle.cuh"
#include "tma.cuh"
#include "track.cuh"

namespace bmadgpu {

namespace {

// One turn's record of a frequency-map job (the per-turn step of frequency_map.f90:288-312):
// the stop test against a quarter RF wavelength, then psv_norm = norm (vec - co). Kept out of
// line so the record's registers do not weigh on the tracking loop of every other variant.
__device__ __noinline__ void fma_record(const BatchVar& v, int64_t j, int32_t t_rel, double x, double px, double y,
                                        double py, double z, double pz) {
  if (v.rec_state[j] != 0) return;
  const double* q = v.rec_par;
  const double psv[6] = {x - q[36], px - q[37], y - q[38], py - q[39], z - q[40], pz - q[41]};
  const double z_limit = q[42];
  if (z_limit > 0 && (fabs(psv[4]) > z_limit || (t_rel == v.rec_turns - 1 && !(fabs(z) < z_limit)))) {
    v.rec_state[j] = 2;
    v.rec_state[v.n + j] = t_rel + 1;
    return;
  }
  const int64_t n = v.n;
  for (int r = 0; r < 6; r++) {
    double s = 0;
    for (int k = 0; k < 6; k++) s = s + q[r * 6 + k] * psv[k];
    v.rec[((int64_t)r * v.rec_turns + t_rel) * n + j] = s;
  }
}

// REC: the instantiation for rounds that hold a frequency-map job; every other launch uses the
// REC = false code, which has no record path at all.
template <int BLOCK, int MINB, bool REC>
__global__ void __launch_bounds__(BLOCK, MINB) k_batch_track(const BatchArgs a, int ppt) {
  extern __shared__ __align__(128) uint8_t smem[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ __align__(16) BatchVar sv;
  __shared__ long long s_item;
  __shared__ int s_var;
  bool can_stage = a.smem_bytes > 0;
  bool pending = false;  // a staging copy whose wait timed out may still be landing
  uint32_t phase = 0;
  if (can_stage && threadIdx.x == 0) mbar_init(&bar, 1);
  int cur_v = -1;
  const uint8_t* tbl = nullptr;
  const long long total = (long long)a.tile_prefix[a.n_var];
  const int lane = threadIdx.x & 31;

  for (;;) {
    if (threadIdx.x == 0) {
      const long long item = (long long)atomicAdd(a.queue, 1ull);
      int v = -1;
      if (item < total) {
        // last variant whose first item is <= item (variants without items share their
        // successor's prefix value and are skipped)
        int lo = 0, hi = a.n_var - 1;
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (a.tile_prefix[mid] <= item) lo = mid;
          else hi = mid - 1;
        }
        v = lo;
      }
      s_item = item;
      s_var = v;
    }
    __syncthreads();
    const long long item = s_item;
    const int v = s_var;
    if (v < 0) break;
    if (v != cur_v) {
      if (threadIdx.x == 0) sv = a.vars[v];
      __syncthreads();
      tbl = sv.table;
      if (can_stage && sv.table_bytes <= a.smem_bytes) {
        if (threadIdx.x == 0) stage_table_issue(smem, sv.table, sv.table_bytes, &bar);
        const bool ok = mbar_wait_bounded(&bar, phase);
        if (__syncthreads_and(ok)) {
          phase ^= 1;
          tbl = smem;
        } else {
          // keep reading the table from global memory; shared memory is not touched again
          if (threadIdx.x == 0) atomicOr(a.err_flag, 1);
          can_stage = false;
          pending = true;
        }
      }
      cur_v = v;
    }

    const EleHdr* hdr = reinterpret_cast<const EleHdr*>(tbl);
    const ApRec* ap = reinterpret_cast<const ApRec*>(tbl + sv.hdr_bytes);
    const double* pool = reinterpret_cast<const double*>(tbl + sv.hdr_bytes + sv.ap_bytes);
    const Globals& G = sv.G;
    const int64_t off = sv.off;
    const SoA soa{a.vec + 6 * off, a.beta + off, a.t ? a.t + off : nullptr, a.state + off,
                  a.ix_ele ? a.ix_ele + off : nullptr, a.ix_turn ? a.ix_turn + off : nullptr,
                  a.location ? a.location + off : nullptr, sv.n};
    const int n_ele = (int)sv.n_ele;
    const int nt = min(a.n_turns, sv.n_turns - a.turn_off);
    const int turn_no0 = sv.turn0 + a.turn_off;
    const double seg_ref = sv.ref_prefix[n_ele] - sv.ref_prefix[0];
    const int64_t n_live = a.live_in ? (int64_t)a.n_in[v] : sv.n;
    const int64_t t0 = (int64_t)(item - a.tile_prefix[v]) * a.tile;

    for (int k = 0; k < ppt; ++k) {
      const int64_t w = t0 + (int64_t)k * BLOCK + threadIdx.x;
      const bool valid = w < n_live;
      const int64_t j = valid ? (a.live_in ? (int64_t)a.live_in[off + w] : w) : 0;
      Particle p;
      p.state = 0;
      if (valid) load_particle(soa, j, p);
      bool alive = valid && p.state == S_ALIVE;
      const double z_in = p.z, beta_in = p.beta;
      LossInfo li;
      if (alive) {
        refresh(p, G);
        for (int turn = 0; turn < nt && alive; ++turn) {
          alive = track_turn(p, hdr, pool, ap, G, 0, n_ele, turn == 0, turn_no0 + turn, li);
          if (REC && sv.rec && alive)
            fma_record(sv, j, turn_no0 + turn - sv.rec_turn0, p.x, p.px, p.y, p.py, p.z, p.pz);
        }
      }
      if (valid) store_particle(soa, j, p, alive, li, z_in, beta_in, nt, turn_no0, seg_ref, sv.ref_prefix, 0);
      if (a.live_out) {
        const unsigned mask = __ballot_sync(0xffffffffu, alive);
        unsigned long long base = 0;
        if (lane == 0 && mask) base = atomicAdd(a.n_out + v, (unsigned long long)__popc(mask));
        base = __shfl_sync(0xffffffffu, base, 0);
        if (alive) a.live_out[off + (int64_t)base + __popc(mask & ((1u << lane) - 1))] = (int32_t)j;
      }
    }
    __syncthreads();  // everyone is done with s_item, sv and the staged table
  }
  if (pending) mbar_wait_bounded(&bar, phase);
}

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
  const void* fn_rec;
};
#define BG_BATCH_VARIANT(B, M) {B, M, (const void*)k_batch_track<B, M, false>, (const void*)k_batch_track<B, M, true>}
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
  if (!v || cfg.particles_per_thread < 1) return cudaErrorInvalidValue;
  cudaError_t err = cudaFuncSetAttribute(v->fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes);
  if (err != cudaSuccess) return err;
  err = cudaFuncSetAttribute(v->fn_rec, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes);
  if (err != cudaSuccess) return err;
  int per_sm = 0;
  err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, v->fn, cfg.block, smem_bytes);
  if (err != cudaSuccess) return err;
  if (per_sm < 1) per_sm = 1;
  int per_sm_rec = 0;
  err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_rec, v->fn_rec, cfg.block, smem_bytes);
  if (err != cudaSuccess) return err;
  if (per_sm_rec < 1) per_sm_rec = 1;
  out->fn = v->fn;
  out->fn_rec = v->fn_rec;
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
  if (record)
    return cudaLaunchKernel(k.fn_rec, dim3((unsigned)k.grid_rec), dim3((unsigned)k.block), args, k.smem, stream);
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
