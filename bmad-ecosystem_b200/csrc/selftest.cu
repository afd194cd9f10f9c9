// selftest.cu -- device self-checks of arithmetic the maps rely on.
//
// k_check_div: the shared-reciprocal quotient div_rcp(a, b, RN(1/b)) (maps.cuh) against the
// device's own division a / b, bit for bit, on n pseudo-random pairs (splitmix64 stream): random
// signs, 52-bit mantissas and exponents in [-60, 60], half of them numerators one ulp either side
// of an exact product b q (quotients next to a rounding tie), plus zero numerators.
// k_cr_eval: the correctly rounded transcendentals of the maps (crmath.cuh) on given arguments,
// for comparison with their host build and with mpmath in the tests.

#define BG_SHARED_RECIPROCAL  // the quotient under test
#include <cuda_runtime.h>

#include <algorithm>

#include "capi_internal.h"
#include "crmath.cuh"
#include "maps.cuh"

using namespace bmadgpu;

namespace {

__device__ inline uint64_t splitmix64(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__device__ inline double random_double(uint64_t& s) {
  const uint64_t r = splitmix64(s);
  const uint64_t mant = r & ((1ull << 52) - 1);
  const int e = (int)((r >> 52) % 121) - 60;
  const uint64_t bits = ((uint64_t)(1023 + e) << 52) | mant;
  const double v = __longlong_as_double((long long)bits);
  return (r >> 63) ? -v : v;
}

__global__ void k_check_div(int64_t n, uint64_t seed, unsigned long long* mismatches) {
  unsigned long long bad = 0;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    uint64_t s = seed ^ ((uint64_t)i * 0xD1B54A32D192ED03ull);
    const double b = random_double(s);
    double a;
    const uint64_t kind = splitmix64(s) % 8;
    if (kind < 4) {
      a = random_double(s);
    } else if (kind < 7) {  // next to an exact product: quotient next to a tie or a representable
      const double q = random_double(s);
      const double p = b * q;
      a = (kind == 4) ? p : (kind == 5 ? nextafter(p, 1e308) : nextafter(p, -1e308));
    } else {
      a = (splitmix64(s) & 1) ? 0.0 : -0.0;
    }
    const double y = 1 / b;
    const double want = a / b, got = div_rcp(a, b, y);
    if (__double_as_longlong(want) != __double_as_longlong(got)) bad++;
  }
  if (bad) atomicAdd(mismatches, bad);
}

__global__ void k_cr_eval(int fn, const double* __restrict__ a, const double* __restrict__ b, double* __restrict__ out,
                          int64_t n) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const double x = a[i];
    double r;
    switch (fn) {
      case 0: r = cr::sin(x); break;
      case 1: r = cr::cos(x); break;
      case 2: r = cr::asin(x); break;
      case 3: r = cr::atan2(x, b[i]); break;
      case 4: r = cr::sinh(x); break;
      case 5: r = cr::cosh(x); break;
      case 8: r = cr::exp(x); break;
      case 9: r = cr::tan(x); break;
      case 6: {  // sincos: sin in out[i], cos in out[n + i]
        double c;
        cr::sincos(x, &r, &c);
        out[n + i] = c;
        break;
      }
      default: {  // sinhcosh
        double c;
        cr::sinhcosh(x, &r, &c);
        out[n + i] = c;
        break;
      }
    }
    out[i] = r;
  }
}

}  // namespace

extern "C" int bmadgpu_cr_eval(bmadgpu_ctx* c, int32_t fn, const double* a, const double* b, double* out, int64_t n) {
  if (!c || !a || !out || n < 0 || fn < 0 || fn > 9 || (fn == 3 && !b)) return fail(BMADGPU_EINVAL, "bad argument");
  CUDA_TRY(cudaSetDevice(c->device));
  if (n == 0) return BMADGPU_OK;
  const int64_t blocks = std::min<int64_t>((n + 255) / 256, (int64_t)c->sm_count * 8);
  k_cr_eval<<<(int)blocks, 256, 0, c->stream>>>(fn, a, b, out, n);
  CUDA_TRY(cudaGetLastError());
  c->launches++;
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  return BMADGPU_OK;
}

extern "C" int bmadgpu_selftest_division(bmadgpu_ctx* c, int64_t n, uint64_t seed, int64_t* mismatches) {
  if (!c || !mismatches || n < 0) return fail(BMADGPU_EINVAL, "bad argument");
  CUDA_TRY(cudaSetDevice(c->device));
  unsigned long long* d = nullptr;
  CUDA_TRY(cudaMalloc(&d, sizeof(unsigned long long)));
  cudaError_t e = cudaMemsetAsync(d, 0, sizeof(unsigned long long), c->stream);
  if (e == cudaSuccess) {
    k_check_div<<<c->sm_count * 8, 256, 0, c->stream>>>(n, seed, d);
    e = cudaGetLastError();
    c->launches++;
  }
  unsigned long long h = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h, d, sizeof(h), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  cudaFree(d);
  if (e != cudaSuccess) return cuda_fail(e, "bmadgpu_selftest_division");
  *mismatches = (int64_t)h;
  return BMADGPU_OK;
}
