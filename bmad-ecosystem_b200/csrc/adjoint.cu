// adjoint.cu -- d(loss)/d(element strengths) on the GPU (bmadgpu_loss_grad of include/bmadgpu.h).
//
// k_adjoint: one thread per particle runs adj_particle (adjoint.cuh): the forward turns with a
// checkpoint every `every` turns, then the reverse sweep, segment by segment from the last
// checkpoint, re-running each segment's turns and each turn's elements so every element's
// vector-Jacobian product sees its own input. Per-particle strength derivatives accumulate in a
// [slot][particle] buffer (each thread owns its column: no atomics).
// k_adj_reduce: one CTA per slot sums the column in a fixed order (deterministic), divides by the
// strength (scale form -> d/dk) and writes the gradient; slot n_slot sums the loss.

#include <cuda_runtime.h>

#include <cstring>
#include <string>
#include <vector>

#include "adjoint.cuh"
#include "capi_internal.h"

using namespace bmadgpu;

namespace bmadgpu {
cudaError_t adjoint_upload_constants();
}

namespace {

constexpr int kAdjBlock = 64;

__global__ void __launch_bounds__(kAdjBlock) k_adjoint(const AdjArgs a) {
  const int64_t j = (int64_t)blockIdx.x * kAdjBlock + threadIdx.x;
  if (j < a.N) adj_particle(a, j);
}

// Sum of row r of a [rows][N] buffer in a fixed order; one CTA of 256 threads per row.
__global__ void k_adj_reduce(const double* __restrict__ gradbuf, const double* __restrict__ lossbuf, int64_t N,
                             int n_slot, const double* __restrict__ strength, double* __restrict__ out) {
  __shared__ double part[256];
  const int r = blockIdx.x;
  const double* row = r < n_slot ? gradbuf + (int64_t)r * N : lossbuf;
  double s = 0;
  for (int64_t j = threadIdx.x; j < N; j += 256) s += row[j];
  part[threadIdx.x] = s;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) part[threadIdx.x] += part[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[r] = r < n_slot ? part[0] / strength[r] : part[0];
}

}  // namespace

namespace bmadgpu {

cudaError_t adjoint_upload_constants() {
  double cm[22][22], cf[22][22];
  build_cmulti_tables(cm, cf);
  cudaError_t e = cudaMemcpyToSymbol(c_cmulti, cm, sizeof(cm));
  if (e != cudaSuccess) return e;
  return cudaMemcpyToSymbol(c_cfull, cf, sizeof(cf));
}

}  // namespace bmadgpu

namespace {

// Device buffers of one call, freed on every return path.
struct AdjBuffers {
  std::vector<void*> ptrs;
  template <class T>
  bool get(T** p, size_t count) {
    void* q = nullptr;
    if (cudaMalloc(&q, count * sizeof(T) + 16) != cudaSuccess) return false;
    ptrs.push_back(q);
    *p = static_cast<T*>(q);
    return true;
  }
  ~AdjBuffers() {
    for (void* p : ptrs) cudaFree(p);
  }
};

// Strength attribute of an element the gradient is taken for, or 0 if it is not a strength
// element; all of the element's field coefficients must scale with it.
int strength_of(const bmadgpu_element& e, double* k, std::string& why) {
  switch (e.key) {
    case BMADGPU_QUADRUPOLE: *k = e.k1; break;
    case BMADGPU_SEXTUPOLE: *k = e.k2; break;
    case BMADGPU_OCTUPOLE: *k = e.k3; break;
    default: why = "gradient element is not a quadrupole, sextupole or octupole"; return BMADGPU_EINVAL;
  }
  if (*k == 0) {
    why = "gradient element has zero strength (the derivative is taken in scale form)";
    return BMADGPU_EINVAL;
  }
  if (e.hkick != 0 || e.vkick != 0) {
    why = "gradient element has hkick/vkick, which do not scale with its strength";
    return BMADGPU_EUNSUPPORTED;
  }
  if (!e.scale_multipoles) {
    for (int n = 0; n < BMADGPU_N_POLE; n++)
      if (e.a_pole[n] != 0 || e.b_pole[n] != 0) {
        why = "gradient element has multipoles not scaled with its strength (scale_multipoles = F)";
        return BMADGPU_EUNSUPPORTED;
      }
  }
  return BMADGPU_OK;
}

}  // namespace

extern "C" int bmadgpu_loss_grad(bmadgpu_ctx* c, const bmadgpu_lattice* lat, const bmadgpu_bunch* b, int32_t n_turns,
                                 int32_t every, int32_t n_param, const int32_t* param_ele, double* loss,
                                 double* grad) {
  if (!c || !lat || !b || !loss || (n_param > 0 && (!param_ele || !grad))) return fail(BMADGPU_EINVAL, "NULL argument");
  if (b->n < 1 || !b->vec || !b->beta || !b->state) return fail(BMADGPU_EINVAL, "bunch is empty or incomplete");
  if (n_turns < 1 || every < 1 || n_param < 0) return fail(BMADGPU_EINVAL, "bad turn count, interval or parameter count");
  if (lat->device != c->device) return fail(BMADGPU_EINVAL, "lattice and context are on different devices");
  const int32_t n_ele = (int32_t)lat->pk.info.n_ele;
  const EleHdr* hdr = reinterpret_cast<const EleHdr*>(lat->pk.image.data());
  for (int32_t i = 0; i < n_ele; i++)
    if (adj_supported(hdr[i]))
      return fail(BMADGPU_EUNSUPPORTED, "element " + std::to_string(i) +
                                            " is outside the adjoint path (edge fringe, bend k1 or multipoles, thin "
                                            "multipole, pitch or z_offset, or more than 16 steps)");
  std::vector<int32_t> slot_of(n_ele, -1);
  std::vector<double> strength(n_param);
  for (int32_t s = 0; s < n_param; s++) {
    const int32_t i = param_ele[s];
    if (i < 0 || i >= n_ele) return fail(BMADGPU_EINVAL, "gradient element index out of range");
    if (slot_of[i] >= 0) return fail(BMADGPU_EINVAL, "gradient element listed twice");
    std::string why;
    int r = strength_of(lat->eles[i], &strength[s], why);
    if (r) return fail(r, why + " (element " + std::to_string(i) + ")");
    slot_of[i] = s;
  }
  CUDA_TRY(cudaSetDevice(c->device));
  const int64_t N = b->n;
  const int32_t n_seg = (n_turns + every - 1) / every;
  AdjBuffers buf;
  double *d_vec, *d_beta, *d_ckpt, *d_turn, *d_ele, *d_grad, *d_loss, *d_strength, *d_out;
  int32_t *d_state, *d_slot;
  const size_t slots = (size_t)(n_param > 0 ? n_param : 1);
  if (!buf.get(&d_vec, 6 * N) || !buf.get(&d_beta, N) || !buf.get(&d_state, N) ||
      !buf.get(&d_ckpt, (size_t)n_seg * 7 * N) || !buf.get(&d_turn, (size_t)every * 7 * N) ||
      !buf.get(&d_ele, (size_t)n_ele * 7 * N) || !buf.get(&d_grad, slots * N) || !buf.get(&d_loss, N) ||
      !buf.get(&d_strength, slots) || !buf.get(&d_out, slots + 1) || !buf.get(&d_slot, (size_t)n_ele))
    return fail(BMADGPU_ENOMEM, "cannot allocate the adjoint's device buffers");
  cudaStream_t s = c->stream;
  CUDA_TRY(cudaMemcpyAsync(d_vec, b->vec, 6 * N * sizeof(double), cudaMemcpyHostToDevice, s));
  CUDA_TRY(cudaMemcpyAsync(d_beta, b->beta, N * sizeof(double), cudaMemcpyHostToDevice, s));
  CUDA_TRY(cudaMemcpyAsync(d_state, b->state, N * sizeof(int32_t), cudaMemcpyHostToDevice, s));
  CUDA_TRY(cudaMemcpyAsync(d_slot, slot_of.data(), n_ele * sizeof(int32_t), cudaMemcpyHostToDevice, s));
  if (n_param > 0)
    CUDA_TRY(cudaMemcpyAsync(d_strength, strength.data(), n_param * sizeof(double), cudaMemcpyHostToDevice, s));
  CUDA_TRY(cudaMemsetAsync(d_grad, 0, slots * N * sizeof(double), s));
  AdjArgs a;
  std::memset(&a, 0, sizeof(a));
  a.hdr = reinterpret_cast<const EleHdr*>(lat->d_table);
  a.ap = reinterpret_cast<const ApRec*>(lat->d_table + lat->pk.info.hdr_bytes);
  a.pool = reinterpret_cast<const double*>(lat->d_table + lat->pk.info.hdr_bytes + lat->pk.info.ap_bytes);
  a.n_ele = n_ele;
  a.n_turns = n_turns;
  a.every = every;
  a.N = N;
  a.G = lat->G;
  a.param_of_ele = d_slot;
  a.ckpt = d_ckpt;
  a.turnbuf = d_turn;
  a.elebuf = d_ele;
  a.gradbuf = d_grad;
  a.lossbuf = d_loss;
  a.vec = d_vec;
  a.beta = d_beta;
  a.state = d_state;
  a.loss_scale = 1.0 / (double)N;
  const unsigned grid = (unsigned)((N + kAdjBlock - 1) / kAdjBlock);
  k_adjoint<<<grid, kAdjBlock, 0, s>>>(a);
  CUDA_TRY(cudaGetLastError());
  k_adj_reduce<<<(unsigned)(n_param + 1), 256, 0, s>>>(d_grad, d_loss, N, n_param, d_strength, d_out);
  CUDA_TRY(cudaGetLastError());
  c->launches += 2;
  std::vector<double> out(n_param + 1);
  CUDA_TRY(cudaMemcpyAsync(out.data(), d_out, (n_param + 1) * sizeof(double), cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  for (int32_t i = 0; i < n_param; i++) grad[i] = out[i];
  *loss = out[n_param];
  return check_err_flag(c);
}
