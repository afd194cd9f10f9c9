// da.cu -- dynamic-aperture search along rays in x-y, all rays at once on the device
// (dynamic_aperture_point, bmad/modules/dynamic_aperture_mod.f90:284-398).
//
// Each ray keeps the reference's search state on the device: the last surviving start point
// (x0, y0), the current trial (x1, y1) and, once bracketed, the lost point (x2, y2). One iteration
// starts every unfinished ray's trial particle (k_da_start), tracks all of them n_turn turns in one
// tracking launch, and updates every ray as the reference's loop does (k_da_update): a loss
// brackets the aperture (turn, element and plane of the loss recorded), survival moves the inner
// point out; the next trial is the midpoint once bracketed, else twice as far; a ray is done when
// the bracket is within 2 (abs_accuracy + r rel_accuracy). The host only reads how many rays are
// still searching.

#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "capi_internal.h"

using namespace bmadgpu;

namespace {

struct RayState {
  double x0, y0, x1, y1, x2, y2;
  int32_t bracketed, done, turn_lost, ix_ele, plane, iterations, failed, pad;
};

__global__ void k_da_init(RayState* rs, const double* __restrict__ theta, int n, double x_init, double y_init) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    RayState r = {};
    r.x1 = cos(theta[i]) * x_init;
    r.y1 = sin(theta[i]) * y_init;
    rs[i] = r;
  }
}

// Trial particles: orbit + (x1, 0, y1, 0, 0, 0) for rays still searching; finished rays get a
// lost state so the tracking skips them.
__global__ void k_da_start(const RayState* __restrict__ rs, const double* __restrict__ orb0, int n, double p0c,
                           double mass, double* vec, double* beta, int32_t* state, int32_t* ix_ele, int32_t* ix_turn,
                           int32_t* location) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const RayState& r = rs[i];
    double v[6];
    for (int k = 0; k < 6; k++) v[k] = orb0 ? orb0[6 * i + k] : 0.0;
    v[0] = v[0] + r.x1;
    v[2] = v[2] + r.y1;
    for (int k = 0; k < 6; k++) vec[k * n + i] = v[k];
    const double pc = p0c * (1 + v[5]);
    beta[i] = pc / sqrt(pc * pc + mass * mass);
    state[i] = r.done ? 2 : 1;
    ix_ele[i] = -1;
    ix_turn[i] = -1;
    location[i] = 0;
  }
}

__global__ void k_da_update(RayState* rs, int n, const int32_t* __restrict__ state, const int32_t* __restrict__ ix_ele,
                            const int32_t* __restrict__ ix_turn, double abs_acc, double rel_acc,
                            unsigned int* n_active) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    RayState r = rs[i];
    if (r.done) continue;
    r.iterations++;
    if (state[i] != 1) {  // lost: the aperture is inside
      r.x2 = r.x1;
      r.y2 = r.y1;
      r.turn_lost = ix_turn[i] + 1;  // the reference counts turns from 1
      r.bracketed = 1;
      r.ix_ele = ix_ele[i];
      r.plane = state[i];
    } else {
      r.x0 = r.x1;
      r.y0 = r.y1;
    }
    if (r.bracketed) {
      r.x1 = (r.x0 + r.x2) / 2;
      r.y1 = (r.y0 + r.y2) / 2;
    } else {
      r.x1 = 2 * r.x1;
      r.y1 = 2 * r.y1;
    }
    if (r.x1 > 1.0 || r.y1 > 1.0) {  // "DA exceeds 1 meter": the reference gives up
      r.failed = 1;
      r.done = 1;
    } else if (r.bracketed) {
      const double rr = 0.5 * sqrt((r.x0 + r.x2) * (r.x0 + r.x2) + (r.y0 + r.y2) * (r.y0 + r.y2));
      if (sqrt((r.x2 - r.x0) * (r.x2 - r.x0) + (r.y2 - r.y0) * (r.y2 - r.y0)) <= 2 * (abs_acc + rr * rel_acc)) r.done = 1;
    }
    rs[i] = r;
    if (!r.done) atomicAdd(n_active, 1u);
  }
}

}  // namespace

extern "C" int bmadgpu_da_scan(bmadgpu_ctx* c, const bmadgpu_lattice* lat, int32_t n_rays, const double* theta,
                               const double* orb0, const bmadgpu_da_params* P, bmadgpu_da_point* out) {
  if (!c || !lat || !P || !out || n_rays < 0 || (n_rays > 0 && !theta)) return fail(BMADGPU_EINVAL, "bad argument");
  if (P->n_turn < 1) return fail(BMADGPU_EINVAL, "n_turn < 1");
  if (lat->device != c->device) return fail(BMADGPU_EINVAL, "lattice and context are on different devices");
  for (int32_t i = 0; i < n_rays; i++) {
    if (P->x_init == 0 && std::fabs(std::cos(theta[i])) > 1e-10) return fail(BMADGPU_EINVAL, "x_init == 0");
    if (P->y_init == 0 && std::fabs(std::sin(theta[i])) > 1e-10) return fail(BMADGPU_EINVAL, "y_init == 0");
  }
  if (n_rays == 0) return BMADGPU_OK;
  CUDA_TRY(cudaSetDevice(c->device));
  const int n = n_rays;
  std::vector<void*> mem;
  struct Free {
    std::vector<void*>& m;
    ~Free() {
      for (void* p : m) cudaFree(p);
    }
  } freer{mem};
  auto get = [&](size_t bytes) -> void* {
    void* p = nullptr;
    if (cudaMalloc(&p, bytes + 16) != cudaSuccess) return nullptr;
    mem.push_back(p);
    return p;
  };
  RayState* rs = (RayState*)get(sizeof(RayState) * n);
  double* d_theta = (double*)get(sizeof(double) * n);
  double* d_orb = orb0 ? (double*)get(sizeof(double) * 6 * n) : nullptr;
  bmadgpu_bunch b;
  b.n = n;
  b.vec = (double*)get(sizeof(double) * 6 * n);
  b.beta = (double*)get(sizeof(double) * n);
  b.t = nullptr;
  b.state = (int32_t*)get(sizeof(int32_t) * n);
  b.ix_ele = (int32_t*)get(sizeof(int32_t) * n);
  b.ix_turn = (int32_t*)get(sizeof(int32_t) * n);
  b.location = (int32_t*)get(sizeof(int32_t) * n);
  unsigned int* d_active = (unsigned int*)get(sizeof(unsigned int));
  if (!rs || !d_theta || (orb0 && !d_orb) || !b.vec || !b.beta || !b.state || !b.ix_ele || !b.ix_turn ||
      !b.location || !d_active)
    return fail(BMADGPU_ENOMEM, "cannot allocate the aperture search state");
  cudaStream_t s = c->stream;
  CUDA_TRY(cudaMemcpyAsync(d_theta, theta, sizeof(double) * n, cudaMemcpyHostToDevice, s));
  if (orb0) CUDA_TRY(cudaMemcpyAsync(d_orb, orb0, sizeof(double) * 6 * n, cudaMemcpyHostToDevice, s));
  const int blocks = (n + 255) / 256;
  k_da_init<<<blocks, 256, 0, s>>>(rs, d_theta, n, P->x_init, P->y_init);
  CUDA_TRY(cudaGetLastError());
  c->launches++;
  const int max_it = P->max_iterations > 0 ? P->max_iterations : 200;
  for (int it = 0; it < max_it; ++it) {
    k_da_start<<<blocks, 256, 0, s>>>(rs, d_orb, n, lat->param.p0c, lat->param.mass, b.vec, b.beta, b.state,
                                       b.ix_ele, b.ix_turn, b.location);
    CUDA_TRY(cudaGetLastError());
    c->launches++;
    int r = track_device(c, lat, &b, 0, (int32_t)lat->pk.info.n_ele, 0, P->n_turn, nullptr);
    if (r) return r;
    CUDA_TRY(cudaMemsetAsync(d_active, 0, sizeof(unsigned int), s));
    k_da_update<<<blocks, 256, 0, s>>>(rs, n, b.state, b.ix_ele, b.ix_turn, P->abs_accuracy, P->rel_accuracy,
                                        d_active);
    CUDA_TRY(cudaGetLastError());
    c->launches++;
    unsigned int active = 0;
    CUDA_TRY(cudaMemcpyAsync(&active, d_active, sizeof(active), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    if (active == 0) break;
  }
  std::vector<RayState> h(n);
  CUDA_TRY(cudaMemcpyAsync(h.data(), rs, sizeof(RayState) * n, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  int failed = 0;
  for (int i = 0; i < n; i++) {
    out[i].x = h[i].x1;
    out[i].y = h[i].y1;
    out[i].i_turn = h[i].turn_lost;
    out[i].ix_ele = h[i].ix_ele;
    out[i].plane = h[i].plane;
    out[i].iterations = h[i].iterations;
    failed += h[i].failed || !h[i].done;
  }
  int r = check_err_flag(c);
  if (r) return r;
  if (failed) return fail(BMADGPU_ETIMEDOUT, "some rays did not converge (aperture beyond 1 m or iteration limit)");
  return BMADGPU_OK;
}
