// track.cuh -- kernel launch interface shared by the C-ABI layer and the kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "table.h"

namespace bmadgpu {

// Arguments of the multi-turn tracking kernel (one thread = one particle).
struct TrackArgs {
  const uint8_t* table;        // packed element table (device)
  uint32_t table_bytes, hdr_bytes, ap_bytes;
  int32_t ix_start, ix_end;    // element range [ix_start, ix_end) tracked each turn
  int32_t turn0, n_turns;
  const int64_t* n_work;       // device: number of particles to work on (live-list length)
  const int32_t* live;         // device: live particle indices, or nullptr for 0 .. n_work-1
  int64_t ld;                  // leading dimension of vec (number of particles in the SoA)
  double* vec;                 // [6][ld]
  double* beta;
  double* t;                   // nullable
  int32_t* state;
  int32_t* ix_ele;             // nullable
  int32_t* ix_turn;            // nullable
  int32_t* location;           // nullable
  double* moments;             // nullable: [n_turns][28]
  const double* ref_prefix;    // [n_ele + 1] sums of delta_ref_time
  Globals G;
  int32_t* err_flag;           // device: bit 0 = table staging wait timed out
  int32_t rare;                // the table has extra blocks / pitched offsets: the full kernel
};

struct LaunchCfg {
  int block = 128;             // threads per CTA
  int ctas_per_sm = 0;         // 0: as many as fit (occupancy), else a cap
  bool stage_smem = true;      // stage the element table in shared memory (TMA bulk copy)
};

int table_fits_smem(uint32_t table_bytes);
cudaError_t upload_constants();
cudaError_t measure_fp64_peak(int sm_count, cudaStream_t stream, double* flops_per_s);
cudaError_t launch_track(const TrackArgs& a, const LaunchCfg& cfg, int sm_count, cudaStream_t stream);

// Warp-ballot stream compaction of the live particles: live_out gets the indices (taken from
// live_in, or 0..n-1) whose state is alive; *n_out receives the count.
cudaError_t launch_compact(const int32_t* state, const int32_t* live_in, const int64_t* n_in, int64_t n_max,
                           int32_t* live_out, int64_t* n_out, cudaStream_t stream);

}  // namespace bmadgpu
