// naff.cu -- NAFF frequency decomposition (naff, sim_utils/math/naff.f90:72-131) of many complex
// signals at once: one CTA per signal, the signal and its windowed copy in shared memory.
//
// Per component, as the reference does: an interpolated-FFT estimate of the spectral peak
// (interpolated_fft_gsl, naff.f90:230-290: Gaussian window r = 8, backward transform -- radix-2
// for power-of-two lengths, a direct sum otherwise -- peak over
// bins 2..N-1, log-parabola interpolation), refined by maximising the Hanning-windowed projection
// |<w s | exp(-2 pi i f t)>| (maximize_projection, naff.f90:160-205) with Brent's method (R. P.
// Brent, Algorithms for Minimization without Derivatives, 1973, ch. 5) from a golden-ratio
// bracket, to the reference's tolerances (relative 1e-8, absolute 1e-15); then the new basis
// vector exp(-2 pi i f t) is orthogonalised against the earlier ones (modified Gram-Schmidt, as
// naff.f90:117-120), its amplitude is the projection of the signal on it, and it is removed from
// the signal.
//
// Every thread runs the same scalar search: the objective is a CTA reduction in a fixed order whose
// result every thread reads from shared memory, so all threads take the same branches. Each thread
// owns the samples t = threadIdx.x + k blockDim.x in every loop over t.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "capi_internal.h"

using namespace bmadgpu;

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kMaxSamples = 4096;  // shared memory: 5 doubles per sample
constexpr double kGold = 1.6180339887498949;
constexpr double kCGold = 0.3819660112501051;

struct Red {
  double a[kWarps], b[kWarps];
};

// (sum a, sum b) over the CTA, the same bits in every thread.
__device__ inline void block_sum2(double& a, double& b, Red& r) {
  for (int off = 16; off > 0; off >>= 1) {
    a += __shfl_down_sync(0xffffffffu, a, off);
    b += __shfl_down_sync(0xffffffffu, b, off);
  }
  __syncthreads();  // earlier readers of r are done
  if ((threadIdx.x & 31) == 0) {
    r.a[threadIdx.x >> 5] = a;
    r.b[threadIdx.x >> 5] = b;
  }
  __syncthreads();
  a = 0;
  b = 0;
  for (int w = 0; w < kWarps; w++) {
    a += r.a[w];
    b += r.b[w];
  }
}

struct Sig {
  double *re, *im, *wre, *wim, *amp;
  const double2* tw;  // exp(+2 pi i m / N), m = 0..N-1 (global, shared by all CTAs)
  int n;
};

// -|<w s | exp(-2 pi i f t)>| = -|sum conj(ws_t) exp(-2 pi i f t)| / N
__device__ double objective(const Sig& s, double f, Red& r) {
  double xr = 0, xi = 0;
  for (int t = threadIdx.x; t < s.n; t += kThreads) {
    double sn, cs;
    sincospi(2.0 * f * t, &sn, &cs);
    // conj(w) * (cs - i sn) = (wr cs - wi sn) - i (wr sn + wi cs)
    xr += s.wre[t] * cs - s.wim[t] * sn;
    xi += -(s.wre[t] * sn + s.wim[t] * cs);
  }
  block_sum2(xr, xi, r);
  return -sqrt(xr * xr + xi * xi) / s.n;
}

// Peak estimate of the Gaussian-windowed spectrum; false if the reference's checks fail.
__device__ bool interpolated_fft(const Sig& s, double* f_out, Red& r) {
  const int n = s.n;
  const double h = (n - 1) / 2.0;
  for (int t = threadIdx.x; t < n; t += kThreads) {
    const double q = 8.0 * ((1.0 * (t + 1)) - h - 1.0) / (n - 1.0);
    const double w = exp(-0.5 * (q * q));
    s.wre[t] = s.re[t] * w;
    s.wim[t] = s.im[t] * w;
  }
  __syncthreads();
  if ((n & (n - 1)) == 0) {
    // power of two: in-place radix-2 transform of the windowed copy (bit reversal, then log2 N
    // butterfly stages with the twiddles exp(+2 pi i pos / len) = w[pos N / len])
    int lg = 0;
    while ((1 << lg) < n) lg++;
    for (int i = threadIdx.x; i < n; i += kThreads) {
      const int rv = (int)(__brev((unsigned)i) >> (32 - lg));
      if (i < rv) {
        const double tr = s.wre[i], ti = s.wim[i];
        s.wre[i] = s.wre[rv];
        s.wim[i] = s.wim[rv];
        s.wre[rv] = tr;
        s.wim[rv] = ti;
      }
    }
    __syncthreads();
    for (int len = 2; len <= n; len <<= 1) {
      const int h = len >> 1, step = n / len;
      for (int t = threadIdx.x; t < n / 2; t += kThreads) {
        const int g = t / h, pos = t - g * h;
        const int ia = g * len + pos, ib = ia + h;
        const double2 w = s.tw[pos * step];
        const double xr = s.wre[ib] * w.x - s.wim[ib] * w.y, xi = s.wre[ib] * w.y + s.wim[ib] * w.x;
        const double ar = s.wre[ia], ai = s.wim[ia];
        s.wre[ib] = ar - xr;
        s.wim[ib] = ai - xi;
        s.wre[ia] = ar + xr;
        s.wim[ia] = ai + xi;
      }
      __syncthreads();
    }
    for (int k = threadIdx.x; k < n; k += kThreads) s.amp[k] = sqrt(s.wre[k] * s.wre[k] + s.wim[k] * s.wim[k]);
  } else {
    for (int k = threadIdx.x; k < n; k += kThreads) {
      double xr = 0, xi = 0;
      int m = 0;  // (j k) mod N
      for (int j = 0; j < n; j++) {
        const double2 w = s.tw[m];  // exp(+2 pi i j k / N)
        xr += s.wre[j] * w.x - s.wim[j] * w.y;
        xi += s.wre[j] * w.y + s.wim[j] * w.x;
        m += k;
        if (m >= n) m -= n;
      }
      s.amp[k] = sqrt(xr * xr + xi * xi);
    }
  }
  __syncthreads();
  __shared__ double sh_f;
  __shared__ int sh_ok;
  if (threadIdx.x == 0) {
    int k = 1;
    for (int j = 2; j < n - 1; j++)
      if (s.amp[j] > s.amp[k]) k = j;  // first maximum over bins 2..N-1
    sh_ok = 0;
    if (s.amp[k] != 0) {
      const double lk = log(s.amp[k]), lkm = log(s.amp[k - 1]), lkp = log(s.amp[k + 1]);
      const double den = 2.0 * lk - lkp - lkm;
      if (den != 0) {
        sh_f = (1.0 * k + (lkp - lkm) / 2.0 / den) / n;
        sh_ok = 1;
      }
    }
  }
  __syncthreads();
  *f_out = sh_f;
  return sh_ok != 0;
}

__device__ double maximize_projection(const Sig& s, double seed, Red& r) {
  const int n = s.n;
  const double h = (n - 1) / 2.0;
  __syncthreads();
  for (int t = threadIdx.x; t < n; t += kThreads) {
    const double w = 0.5 * (1.0 + cospi(2.0 * ((t + 1) - h - 1) / (n - 1)));
    s.wre[t] = s.re[t] * w;
    s.wim[t] = s.im[t] * w;
  }
  __syncthreads();
  // golden-ratio bracket from (seed, seed + 0.1 / N), downhill
  double a = seed, b = seed + 0.1 / n;
  double fa = objective(s, a, r), fb = objective(s, b, r);
  if (fb > fa) {
    double t = a;
    a = b;
    b = t;
    t = fa;
    fa = fb;
    fb = t;
  }
  double c = b + kGold * (b - a), fc = objective(s, c, r);
  for (int it = 0; it < 200 && fc < fb; it++) {
    a = b;
    fa = fb;
    b = c;
    fb = fc;
    c = b + kGold * (b - a);
    fc = objective(s, c, r);
  }
  // Brent's minimisation inside [min(a, c), max(a, c)] starting from b
  double lo = fmin(a, c), hi = fmax(a, c);
  double x = b, w = b, v = b, fx = fb, fw = fb, fv = fb, d = 0, e = 0;
  for (int it = 0; it < 100; it++) {
    const double mid = 0.5 * (lo + hi);
    const double tol1 = 1e-8 * fabs(x) + 1e-15, tol2 = 2.0 * tol1;
    if (fabs(x - mid) <= tol2 - 0.5 * (hi - lo)) break;
    bool golden = true;
    if (fabs(e) > tol1) {
      const double rr = (x - w) * (fx - fv);
      double q = (x - v) * (fx - fw);
      double p = (x - v) * q - (x - w) * rr;
      q = 2.0 * (q - rr);
      if (q > 0) p = -p;
      q = fabs(q);
      const double e_old = e;
      e = d;
      if (fabs(p) < fabs(0.5 * q * e_old) && p > q * (lo - x) && p < q * (hi - x)) {
        d = p / q;
        const double u = x + d;
        if (u - lo < tol2 || hi - u < tol2) d = copysign(tol1, mid - x);
        golden = false;
      }
    }
    if (golden) {
      e = (x >= mid) ? (lo - x) : (hi - x);
      d = kCGold * e;
    }
    const double u = fabs(d) >= tol1 ? x + d : x + copysign(tol1, d);
    const double fu = objective(s, u, r);
    if (fu <= fx) {
      if (u >= x)
        lo = x;
      else
        hi = x;
      v = w;
      fv = fw;
      w = x;
      fw = fx;
      x = u;
      fx = fu;
    } else {
      if (u < x)
        lo = u;
      else
        hi = u;
      if (fu <= fw || w == x) {
        v = w;
        fv = fw;
        w = u;
        fw = fu;
      } else if (fu <= fv || v == x || v == w) {
        v = u;
        fv = fu;
      }
    }
  }
  return x;
}

__global__ void k_twiddle(double2* __restrict__ tw, int n) {
  for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < n; m += gridDim.x * blockDim.x) {
    double sn, cs;
    sincospi(2.0 * m / n, &sn, &cs);
    tw[m] = make_double2(cs, sn);
  }
}

__global__ void __launch_bounds__(kThreads) k_naff(const double* __restrict__ cdata, int n, int n_comp, int zero_first,
                                                   const double2* __restrict__ tw, double* __restrict__ ubuf,
                                                   double* __restrict__ freqs, double* __restrict__ amps) {
  extern __shared__ double sm[];
  __shared__ Red red;
  const int64_t sig = blockIdx.x;
  Sig s{sm, sm + n, sm + 2 * n, sm + 3 * n, sm + 4 * n, tw, n};
  const double* src = cdata + sig * 2 * n;
  double* u = ubuf + sig * (int64_t)n_comp * 2 * n;  // [n_comp][n][2]
  double* fo = freqs + sig * n_comp;
  double* ao = amps + sig * n_comp * 2;
  for (int t = threadIdx.x; t < n; t += kThreads) {
    s.re[t] = src[2 * t];
    s.im[t] = src[2 * t + 1];
  }
  __syncthreads();
  int diff = 0;
  for (int t = threadIdx.x; t < n; t += kThreads) diff |= (s.re[t] != s.re[0] || s.im[t] != s.im[0]);
  const bool all_equal = __syncthreads_or(diff) == 0;
  if (threadIdx.x == 0)
    for (int i = 0; i < n_comp; i++) {
      fo[i] = all_equal ? 0.0 : -1.0;
      ao[2 * i] = 0;
      ao[2 * i + 1] = 0;
    }
  if (all_equal) return;
  for (int i = 0; i < n_comp; i++) {
    double f;
    if (i == 0 && zero_first) {
      f = 0.0;
    } else {
      if (!interpolated_fft(s, &f, red)) return;
      f = maximize_projection(s, f, red);
    }
    double* ui = u + (int64_t)i * 2 * n;
    for (int t = threadIdx.x; t < n; t += kThreads) {
      double sn, cs;
      sincospi(2.0 * f * t, &sn, &cs);  // exp(-2 pi i f t)
      ui[2 * t] = cs;
      ui[2 * t + 1] = -sn;
    }
    for (int j = 0; j < i; j++) {  // u_i -= <u_j | u_i> u_j
      const double* uj = u + (int64_t)j * 2 * n;
      double pr = 0, pi = 0;
      for (int t = threadIdx.x; t < n; t += kThreads) {
        const double ar = uj[2 * t], ai = uj[2 * t + 1], br = ui[2 * t], bi = ui[2 * t + 1];
        pr += ar * br + ai * bi;  // conj(a) b
        pi += ar * bi - ai * br;
      }
      block_sum2(pr, pi, red);
      pr /= n;
      pi /= n;
      for (int t = threadIdx.x; t < n; t += kThreads) {
        const double ar = uj[2 * t], ai = uj[2 * t + 1];
        ui[2 * t] = ui[2 * t] - (pr * ar - pi * ai);
        ui[2 * t + 1] = ui[2 * t + 1] - (pr * ai + pi * ar);
      }
    }
    double cr = 0, ci = 0;  // amp = <u_i | s>
    for (int t = threadIdx.x; t < n; t += kThreads) {
      const double ar = ui[2 * t], ai = ui[2 * t + 1], br = s.re[t], bi = s.im[t];
      cr += ar * br + ai * bi;
      ci += ar * bi - ai * br;
    }
    block_sum2(cr, ci, red);
    cr /= n;
    ci /= n;
    for (int t = threadIdx.x; t < n; t += kThreads) {
      const double ar = ui[2 * t], ai = ui[2 * t + 1];
      s.re[t] = s.re[t] - (cr * ar - ci * ai);
      s.im[t] = s.im[t] - (cr * ai + ci * ar);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      fo[i] = f;
      ao[2 * i] = cr;
      ao[2 * i + 1] = ci;
    }
  }
}

}  // namespace

extern "C" int bmadgpu_naff(bmadgpu_ctx* c, int32_t n_signals, int32_t n_samples, const double* cdata, int32_t n_comp,
                            int32_t zero_first, double* freqs, double* amps) {
  if (!c || n_signals < 0 || n_comp < 1 || (n_signals > 0 && (!cdata || !freqs || !amps)))
    return fail(BMADGPU_EINVAL, "bad argument");
  if (n_samples < 4 || n_samples > kMaxSamples) return fail(BMADGPU_EINVAL, "n_samples must be in [4, 4096]");
  if (n_signals == 0) return BMADGPU_OK;
  CUDA_TRY(cudaSetDevice(c->device));
  cudaStream_t s = c->stream;
  const size_t data_b = sizeof(double) * 2 * (size_t)n_samples * n_signals;
  const size_t u_b = data_b * n_comp;
  const size_t f_b = sizeof(double) * (size_t)n_signals * n_comp;
  void* mem = nullptr;
  const size_t tw_b = sizeof(double2) * (size_t)n_samples;
  if (cudaMalloc(&mem, data_b + u_b + 3 * f_b + tw_b) != cudaSuccess)
    return fail(BMADGPU_ENOMEM, "cannot allocate NAFF scratch");
  struct Free {
    void* p;
    ~Free() { cudaFree(p); }
  } freer{mem};
  // the twiddle table first: double2 loads need 16-byte alignment
  double2* d_tw = (double2*)mem;
  double* d_data = (double*)(d_tw + n_samples);
  double* d_u = d_data + 2 * (size_t)n_samples * n_signals;
  double* d_f = d_u + 2 * (size_t)n_samples * n_signals * n_comp;
  double* d_a = d_f + (size_t)n_signals * n_comp;
  CUDA_TRY(cudaMemcpyAsync(d_data, cdata, data_b, cudaMemcpyHostToDevice, s));
  const size_t smem = sizeof(double) * 5 * n_samples;
  if (smem > 48 * 1024) CUDA_TRY(cudaFuncSetAttribute(k_naff, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_twiddle<<<(n_samples + 255) / 256, 256, 0, s>>>(d_tw, n_samples);
  CUDA_TRY(cudaGetLastError());
  k_naff<<<n_signals, kThreads, smem, s>>>(d_data, n_samples, n_comp, zero_first, d_tw, d_u, d_f, d_a);
  CUDA_TRY(cudaGetLastError());
  c->launches += 2;
  CUDA_TRY(cudaMemcpyAsync(freqs, d_f, f_b, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaMemcpyAsync(amps, d_a, 2 * f_b, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  return BMADGPU_OK;
}
