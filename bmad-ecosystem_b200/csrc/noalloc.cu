// noalloc.cu -- multi-turn tracking with loss compaction that allocates no memory.
//
// Some callers cannot call cudaMalloc while they track: a host program that gives the GPU's
// memory to its own pool allocator and forbids other allocations during a run, or a loop that
// may not stall on an allocation (cudaMalloc can synchronise the device). bmadgpu_track_bunch_device_noalloc serves them. It runs the
// same tracking and compaction kernels as bmadgpu_track_bunch_device with compaction on, but its
// scratch memory -- the two live-particle index lists and their lengths -- lives in the fixed
// file-scope device array below instead of context buffers grown with cudaMalloc.
//
// Limits and sharing: at most BMADGPU_NOALLOC_MAX_PARTICLES particles per call. The array exists
// once per device that loads this library and stays allocated until the process exits. Every
// call on a device uses the same array and finds there what the previous call left; the lengths
// are reset by each call before use. Calls whose work overlaps on the GPU (two streams, or two
// host threads) race on the array and must be serialised by the caller.

#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "../../include/bmadgpu.h"
#include "track.cuh"

using namespace bmadgpu;

namespace {

// Scratch layout: [0, 256) the two int64 live-list lengths; then the two int32 index lists.
constexpr size_t kLenBytes = 256;
constexpr size_t kListBytes = (size_t)BMADGPU_NOALLOC_MAX_PARTICLES * sizeof(int32_t);
constexpr size_t kScratchBytes = kLenBytes + 2 * kListBytes;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

__global__ void k_noalloc_set_len(int64_t* p, int64_t v) { *p = v; }

// Device address of g_noalloc_scratch per device, looked up once with that device current.
std::mutex g_mu;
void* g_addr[64] = {nullptr};

}  // namespace

namespace bmadgpu {
// Defined in capi.cu: error reporting and argument checks shared with the other entry points.
int noalloc_fail(int code, const char* msg);
int noalloc_prepare(bmadgpu_ctx* ctx, const bmadgpu_lattice* lat, const bmadgpu_bunch* b, TrackArgs* a,
                    LaunchCfg* cfg, int* sm_count, cudaStream_t* stream, int64_t** launches);
}  // namespace bmadgpu

extern "C" int bmadgpu_track_bunch_device_noalloc(bmadgpu_ctx* ctx, const bmadgpu_lattice* lat, bmadgpu_bunch* b,
                                                  int32_t turn0, int32_t n_turns, int32_t turns_per_launch) {
  if (!b) return noalloc_fail(BMADGPU_EINVAL, "bunch is NULL");
  if (b->n > BMADGPU_NOALLOC_MAX_PARTICLES)
    return noalloc_fail(BMADGPU_EINVAL,
                                         "bmadgpu_track_bunch_device_noalloc: more particles than "
                                         "BMADGPU_NOALLOC_MAX_PARTICLES (262144)");
  if (n_turns < 0 || turns_per_launch < 0) return noalloc_fail(BMADGPU_EINVAL, "negative turn count");
  TrackArgs a;
  LaunchCfg cfg;
  int sm_count = 0;
  cudaStream_t s = nullptr;
  int64_t* launches_inc = nullptr;
  int r = noalloc_prepare(ctx, lat, b, &a, &cfg, &sm_count, &s, &launches_inc);
  if (r) return r;
  if (b->n == 0 || n_turns == 0) return BMADGPU_OK;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64)
    return noalloc_fail(BMADGPU_ECUDA, "cudaGetDevice failed");
  unsigned char* base;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[dev]) {
      void* p = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess) return noalloc_fail(BMADGPU_ECUDA, cudaGetErrorString(e));
      g_addr[dev] = p;
    }
    base = (unsigned char*)g_addr[dev];
  }
  int64_t* lens = (int64_t*)base;
  int32_t* lists[2] = {(int32_t*)(base + kLenBytes), (int32_t*)(base + kLenBytes + kListBytes)};

  const int per_launch = turns_per_launch > 0 ? turns_per_launch : n_turns;
  k_noalloc_set_len<<<1, 1, 0, s>>>(lens, b->n);
  if (cudaGetLastError() != cudaSuccess) return noalloc_fail(BMADGPU_ECUDA, "launch failed");
  (*launches_inc)++;
  const int32_t* live = nullptr;
  int cur = 0;
  for (int32_t done = 0; done < n_turns; done += per_launch) {
    int32_t nt = per_launch < n_turns - done ? per_launch : n_turns - done;
    a.turn0 = turn0 + done;
    a.n_turns = nt;
    a.n_work = lens + cur;
    a.live = live;
    a.moments = nullptr;
    cudaError_t e = launch_track(a, cfg, sm_count, s);
    if (e != cudaSuccess) return noalloc_fail(BMADGPU_ECUDA, cudaGetErrorString(e));
    (*launches_inc)++;
    if (done + nt < n_turns) {
      int nxt = live ? 1 - cur : 1;
      e = launch_compact(b->state, live, lens + cur, b->n, lists[nxt], lens + nxt, s);
      if (e != cudaSuccess) return noalloc_fail(BMADGPU_ECUDA, cudaGetErrorString(e));
      (*launches_inc)++;
      live = lists[nxt];
      cur = nxt;
    }
  }
  return BMADGPU_OK;
}
