// capi_internal.h -- context and lattice objects shared by the C-ABI translation units.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/bmadgpu.h"
#include "lattice.h"
#include "track.cuh"

struct bmadgpu_ctx;

namespace bmadgpu {
int fail(int code, const std::string& msg);
int cuda_fail(cudaError_t e, const char* what);
Globals make_globals(const bmadgpu_param& p);
// Reads and clears the context's device error flag (synchronises the context stream).
int check_err_flag(bmadgpu_ctx* c);
// Enqueues n_turns of tracking of a device-resident bunch on the context stream with the
// context's tuning (chunks of turns_per_launch, live-list compaction between them); d_moments,
// if not NULL, receives the per-turn sums [n_turns][28].
int track_device(bmadgpu_ctx* c, const bmadgpu_lattice* lat, const bmadgpu_bunch* b, int32_t ix_start,
                 int32_t ix_end, int32_t turn0, int32_t n_turns, double* d_moments);
// Frequency-map tunes of n particles from their record hist [6][n_turn][n] (fma.cu): fstate[i]
// = 1 where state[i] is not alive, else rec_state[i]; tunes [n][6] where fstate is 0.
cudaError_t fma_launch_tunes(const double* hist, int64_t n, int32_t n_turn, int32_t N, const int32_t* state,
                             const int32_t* rec_state, int32_t* fstate, int32_t flip_a, int32_t flip_b, double* tunes,
                             int sm_count, cudaStream_t s);
}  // namespace bmadgpu

#define CUDA_TRY(call)                                            \
  do {                                                            \
    cudaError_t e_ = (call);                                      \
    if (e_ != cudaSuccess) return bmadgpu::cuda_fail(e_, #call);  \
  } while (0)

struct bmadgpu_ctx {
  int device = 0;
  int sm_count = 0;
  cudaStream_t stream = nullptr;
  int32_t* d_err = nullptr;
  int64_t* d_nwork = nullptr;     // [2] live-list lengths
  int32_t* d_live[2] = {nullptr, nullptr};
  int64_t live_cap = 0;
  // staging for the host-pointer API
  int64_t cap = 0;
  double* d_vec = nullptr;
  double* d_beta = nullptr;
  double* d_t = nullptr;
  double* d_mom = nullptr;
  int64_t mom_cap = 0;
  int32_t* d_i32 = nullptr;       // state, ix_ele, ix_turn, location: 4 * cap
  bmadgpu_tuning tuning;
  int64_t launches = 0;           // kernel launches enqueued
  // autotuner trial copies
  int64_t tune_cap = 0;
  double* d_tvec = nullptr;
  double* d_tbeta = nullptr;
  int32_t* d_tstate = nullptr;
};

struct bmadgpu_lattice {
  int device = 0;
  bmadgpu::PackedLattice pk;
  uint8_t* d_table = nullptr;
  double* d_prefix = nullptr;
  bmadgpu::Globals G;
  bmadgpu_param param;
  std::vector<bmadgpu_element> eles;  // the element records as given (attribute look-ups)
};

