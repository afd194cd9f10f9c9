// batch.cuh -- kernel interface of batched tracking over many lattice variants (batch.cu), used
// by the batch entry points and the serving loop.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "table.h"

namespace bmadgpu {

// Per-variant descriptor in device memory (one lattice + its particles).
struct BatchVar {
  const uint8_t* table;       // packed element table
  const double* ref_prefix;   // [n_ele + 1] sums of delta_ref_time
  int64_t n;                  // particles of the variant
  int64_t off;                // index of its first particle in the batch-wide arrays
  uint32_t table_bytes, hdr_bytes, ap_bytes, n_ele;
  int32_t turn0;              // turn number of call-relative turn 0
  int32_t n_turns;            // turns of the current call for this variant
  Globals G;
  // Frequency-map job (serving): after every turn the normalised coordinates of each surviving
  // particle go to rec [6][rec_turns][n]; nullptr for every other variant.
  double* rec;
  const double* rec_par;      // norm [36] (row-major), closed orbit [6], z_limit (0: no z cut)
  int32_t* rec_state;         // [n] 0 recording, 2 stopped outside the RF bucket; [n, 2n) its turn
  int32_t rec_turn0;          // turn number of the job's first turn
  int32_t rec_turns;          // the job's turn count
};

// Arguments of one launch of k_batch_track: call-relative turns [turn_off, turn_off + n_turns),
// clipped per variant to its n_turns.
struct BatchArgs {
  const BatchVar* vars;
  int32_t n_var;
  int32_t tile;               // particles per work item (threads per CTA x particles per thread)
  double* vec;                // variant v: [6][n_v] block at vec + 6 * off_v
  double* beta;
  double* t;
  int32_t* state;
  int32_t* ix_ele;
  int32_t* ix_turn;
  int32_t* location;
  int32_t turn_off, n_turns;
  const int64_t* tile_prefix;        // [n_var + 1]: first work item of each variant
  const int32_t* live_in;            // variant v's live list at live_in + off_v; nullptr: 0 .. n_v-1
  const unsigned long long* n_in;    // [n_var] live-list lengths (unused with live_in == nullptr)
  int32_t* live_out;                 // nullptr: no compaction after this launch
  unsigned long long* n_out;         // [n_var] lengths of the compacted lists
  unsigned long long* queue;         // work-item counter, zero at launch
  int32_t* err_flag;                 // bit 0: table staging wait timed out
  uint32_t smem_bytes;               // dynamic shared memory for staging (0: read tables from global)
  int32_t rare;                      // some variant's table has extra blocks / pitched offsets
};

struct BatchLaunch {
  int block = 128;
  int ctas_per_sm = 0;        // register budget selector, as LaunchCfg::ctas_per_sm
  int particles_per_thread = 1;
};

// Kernel + grid of a launch shape (resolved once, outside stream capture).
struct BatchKernel {
  const void* fn = nullptr;
  int block = 0, grid = 0, ppt = 1;
  uint32_t smem = 0;
  const void* fn_rec = nullptr;  // the same shape with the frequency-map record path
  int grid_rec = 0;
  const void* fn_lean = nullptr; // the same shape for tables without rare forms (TableInfo::rare)
  int grid_lean = 0;
  const void* fn_rec_lean = nullptr;
  int grid_rec_lean = 0;
};

cudaError_t batch_upload_constants();
cudaError_t batch_rec_upload_constants();            // batch_rec.cu's copy of the tables
// record-path instantiation of a shape (full: every element form; else the lean one)
const void* batch_rec_kernel(int block, int minb, bool full = true);
cudaError_t batch_resolve(const BatchLaunch& cfg, uint32_t smem_bytes, int sm_count, BatchKernel* out);
// record: use the instantiation with the frequency-map record path (rounds with an FMA job).
cudaError_t batch_launch_track(const BatchKernel& k, const BatchArgs& a, cudaStream_t stream, bool record = false);
// Work plan for a launch: tile_prefix from the live counts (or the variants' sizes when
// identity is set), restricted to variants with turns left after turn_off; zeroes the queue
// counter and the next launch's counts (n_zero, nullable).
cudaError_t batch_launch_plan(const BatchVar* vars, int32_t n_var, int32_t tile, int32_t turn_off, bool identity,
                              const unsigned long long* n_in, int64_t* tile_prefix, unsigned long long* queue,
                              unsigned long long* n_zero, cudaStream_t stream);
// Sets turn0 and n_turns of every variant (the batch entry point's per-call values).
cudaError_t batch_launch_set_turns(BatchVar* vars, int32_t n_var, int32_t turn0, int32_t n_turns,
                                   cudaStream_t stream);

// A job's first live list: list[i] = i for i < n, *count = n.
cudaError_t batch_launch_init_list(int32_t* list, int64_t n, unsigned long long* count, cudaStream_t stream);

}  // namespace bmadgpu
