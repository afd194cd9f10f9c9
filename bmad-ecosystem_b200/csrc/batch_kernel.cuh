// batch_kernel.cuh -- the batched tracking kernel k_batch_track (description in batch.cu). Its
// plain instantiations are compiled in batch.cu and the ones with the frequency-map record path
// in batch_rec.cu, so the two compile in parallel.
#pragma once
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
template <int BLOCK, int MINB, bool REC, bool FULL = true>
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
          alive = track_turn<FULL>(p, hdr, pool, ap, G, 0, n_ele, turn == 0, turn_no0 + turn, li);
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

}  // namespace

}  // namespace bmadgpu
