// fma.cu -- frequency-map analysis of many particles at once (bsim/frequency_map/frequency_map.f90:
// 197-376): every particle starts at the closed orbit plus its grid offset, is tracked n_turn
// turns, and its normalised turn-by-turn coordinates give three tunes for the first fft_turns turns
// and three for the last fft_turns turns.
//
// Device layout. The turn-by-turn record is hist[6][n_turn][n] (coordinate, turn, particle), so the
// per-turn record kernel writes coalesced rows. The tune kernel gives one CTA to one signal -- a
// (particle, plane, half) triple, six per particle -- stages its fft_turns Hanning-windowed complex
// samples and a twiddle table of exp(+2 pi i m / N) in shared memory, evaluates the amplitude
// spectrum |X_k| = |sum_j s_j exp(+2 pi i j k / N)| (FFTW_BACKWARD's sign; a radix-2 FFT in shared
// memory for power-of-two N, else a direct transform with the tabulated twiddle w[(j k) mod N], so
// any N works), finds the first
// maximum as the reference's loop does, and applies calc_tune's interpolation
// (frequency_map.f90:364-375). The reference's own turn loop stops a particle when it is lost or,
// with z_cut, when |z - z_co| exceeds a quarter RF wavelength (frequency_map.f90:290-299); here the
// particle is marked at that turn and its tunes are not computed.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "capi_internal.h"

using namespace bmadgpu;

namespace {

constexpr double kCLight = 299792458.0;
constexpr int kTuneThreads = 256;
constexpr int kMaxFftTurns = 4096;  // shared memory: 2 * 16 B * N = 128 KB at the limit

// Normalised coordinates of every particle after `turn` (0-based) into hist, and the stop marks.
__global__ void k_fma_record(const double* __restrict__ vec, const int32_t* __restrict__ state,
                             const int32_t* __restrict__ ix_ele, int64_t n, int32_t turn, int32_t n_turn,
                             const double* __restrict__ norm, const double* __restrict__ co, double z_limit,
                             double* __restrict__ hist, int32_t* __restrict__ fstate, int32_t* __restrict__ fturn,
                             int32_t* __restrict__ fele) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    if (fstate[i] != 0) continue;
    if (state[i] != BMADGPU_ALIVE) {
      fstate[i] = 1;
      fturn[i] = turn + 1;
      fele[i] = ix_ele ? ix_ele[i] : -1;
      continue;
    }
    double psv[6];
    for (int k = 0; k < 6; k++) psv[k] = vec[k * n + i] - co[k];
    if (z_limit > 0 && fabs(psv[4]) > z_limit) {
      fstate[i] = 2;
      fturn[i] = turn + 1;
      continue;
    }
    // after the last turn the reference also wants |z| itself inside the quarter wavelength
    // (frequency_map.f90:327)
    if (z_limit > 0 && turn == n_turn - 1 && !(fabs(vec[4 * n + i]) < z_limit)) {
      fstate[i] = 2;
      fturn[i] = turn + 1;
      continue;
    }
    for (int r = 0; r < 6; r++) {
      double s = 0;
      for (int k = 0; k < 6; k++) s = s + norm[r * 6 + k] * psv[k];
      hist[((int64_t)r * n_turn + turn) * n + i] = s;
    }
  }
}

__device__ inline bool better(double a, int ia, double b, int ib) { return a > b || (a == b && ia < ib); }

// One CTA per signal: blockIdx.x = (particle * 3 + plane) * 2 + half.
__global__ void __launch_bounds__(kTuneThreads) k_fma_tunes(const double* __restrict__ hist, int64_t n, int32_t n_turn,
                                                            int32_t N, const int32_t* __restrict__ fstate,
                                                            int32_t flip_a, int32_t flip_b, double* __restrict__ tunes) {
  extern __shared__ double sm[];
  double* sre = sm;            // [N] windowed samples
  double* sim = sm + N;
  double* wre = sm + 2 * N;    // [N] twiddles
  double* wim = sm + 3 * N;
  __shared__ double best_v[kTuneThreads / 32];
  __shared__ int best_i[kTuneThreads / 32];
  const int64_t sig = blockIdx.x;
  const int64_t p = sig / 6;
  const int plane = (int)((sig / 2) % 3), half = (int)(sig % 2);
  if (fstate[p] != 0) return;  // uniform across the CTA
  const int j0 = half ? n_turn - N : 0;
  const int cre = 2 * plane, cim = 2 * plane + 1;
  const double sgn = plane == 2 ? -1.0 : 1.0;  // n3 = cmplx(z, -pz)
  for (int j = threadIdx.x; j < N; j += blockDim.x) {
    const double s = sinpi((double)(j + 1) / N);
    const double hann = 2 * (s * s);  // 2 sin^2(pi j / N), j counted from 1
    sre[j] = hist[((int64_t)cre * n_turn + j0 + j) * n + p] * hann;
    sim[j] = sgn * hist[((int64_t)cim * n_turn + j0 + j) * n + p] * hann;
    double sn, cs;
    sincospi(2.0 * j / N, &sn, &cs);
    wre[j] = cs;
    wim[j] = sn;
  }
  __syncthreads();
  // A power-of-two N takes an in-place radix-2 transform (bit reversal, then log2 N butterfly
  // stages with the twiddles exp(+2 pi i pos / len) = w[pos N / len]); any other N the direct sum.
  const bool pow2 = (N & (N - 1)) == 0;
  if (pow2) {
    int lg = 0;
    while ((1 << lg) < N) lg++;
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
      const int r = (int)(__brev((unsigned)i) >> (32 - lg));
      if (i < r) {
        const double tr = sre[i], ti = sim[i];
        sre[i] = sre[r];
        sim[i] = sim[r];
        sre[r] = tr;
        sim[r] = ti;
      }
    }
    __syncthreads();
    for (int len = 2; len <= N; len <<= 1) {
      const int h = len >> 1, step = N / len;
      for (int t = threadIdx.x; t < N / 2; t += blockDim.x) {
        const int g = t / h, pos = t - g * h;
        const int ia = g * len + pos, ib = ia + h;
        const double wr = wre[pos * step], wi = wim[pos * step];
        const double xr = sre[ib] * wr - sim[ib] * wi, xi = sre[ib] * wi + sim[ib] * wr;
        const double ar = sre[ia], ai = sim[ia];
        sre[ib] = ar - xr;
        sim[ib] = ai - xi;
        sre[ia] = ar + xr;
        sim[ia] = ai + xi;
      }
      __syncthreads();
    }
  }
  double bv = -1.0;
  int bi = 0;
  for (int k = threadIdx.x; k < N; k += blockDim.x) {
    double xr = 0, xi = 0;
    if (pow2) {
      xr = sre[k];
      xi = sim[k];
    } else {
      int m = 0;  // (j k) mod N, advanced by k each step
      for (int j = 0; j < N; j++) {
        const double a = sre[j], b = sim[j], c = wre[m], d = wim[m];
        xr += a * c - b * d;
        xi += a * d + b * c;
        m += k;
        if (m >= N) m -= N;
      }
    }
    const double amp = sqrt(xr * xr + xi * xi);
    if (better(amp, k, bv, bi)) {
      bv = amp;
      bi = k;
    }
  }
  // CTA arg-max, first index on ties (the reference's strict < scan)
  for (int off = 16; off > 0; off >>= 1) {
    const double ov = __shfl_down_sync(0xffffffffu, bv, off);
    const int oi = __shfl_down_sync(0xffffffffu, bi, off);
    if (better(ov, oi, bv, bi)) {
      bv = ov;
      bi = oi;
    }
  }
  if ((threadIdx.x & 31) == 0) {
    best_v[threadIdx.x >> 5] = bv;
    best_i[threadIdx.x >> 5] = bi;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double v = best_v[0];
    int ix = best_i[0];
    for (int w = 1; w < kTuneThreads / 32; w++)
      if (better(best_v[w], best_i[w], v, ix)) {
        v = best_v[w];
        ix = best_i[w];
      }
    // b = |X| at the next bin (recomputed; 0 past the last bin)
    double b = 0;
    if (ix + 1 < N && pow2) {
      b = sqrt(sre[ix + 1] * sre[ix + 1] + sim[ix + 1] * sim[ix + 1]);
    } else if (ix + 1 < N) {
      double xr = 0, xi = 0;
      int m = 0;
      for (int j = 0; j < N; j++) {
        xr += sre[j] * wre[m] - sim[j] * wim[m];
        xi += sre[j] * wim[m] + sim[j] * wre[m];
        m += ix + 1;
        if (m >= N) m -= N;
      }
      b = sqrt(xr * xr + xi * xi);
    }
    const double d = v;
    const double c = cospi(2.0 / N);
    const double A = (-(d + b * c) * (d - b) + b * sqrt(c * c * (d + b) * (d + b) - 2 * d * b * (2 * c * c - c - 1))) /
                     (d * d + b * b + 2 * d * b * c);
    const int iq = ix + 1;  // 1-based bin as in calc_tune
    double tune = (double)iq / N + (1.0 / (2 * M_PI)) * asin(A * sinpi(2.0 / N));
    if ((plane == 0 && flip_a) || (plane == 1 && flip_b)) tune = 1. - tune;
    tunes[p * 6 + half * 3 + plane] = tune;
  }
}

__global__ void k_fma_start(const double* __restrict__ off, const double* __restrict__ co, int64_t n, double p0c,
                            double e_tot, double mass, double* __restrict__ vec, double* __restrict__ beta,
                            int32_t* __restrict__ state, int32_t* __restrict__ ix_ele, int32_t* __restrict__ ix_turn,
                            int32_t* __restrict__ location, int32_t* __restrict__ fstate) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    for (int k = 0; k < 6; k++) vec[k * n + i] = co[k] + off[i * 6 + k];
    const double pz = vec[5 * n + i];
    if (pz == 0) {
      beta[i] = p0c / e_tot;
    } else {
      const double pc = p0c * (1 + pz);
      beta[i] = pc / sqrt(pc * pc + mass * mass);
    }
    state[i] = BMADGPU_ALIVE;
    ix_ele[i] = -1;
    ix_turn[i] = -1;
    location[i] = 0;
    fstate[i] = 0;
  }
}

__global__ void k_fma_status(const int32_t* __restrict__ state, const int32_t* __restrict__ rec_state, int64_t n,
                             int32_t* __restrict__ fstate) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
    fstate[i] = state[i] != BMADGPU_ALIVE ? 1 : rec_state[i];
}

}  // namespace

namespace bmadgpu {

cudaError_t fma_launch_tunes(const double* hist, int64_t n, int32_t n_turn, int32_t N, const int32_t* state,
                             const int32_t* rec_state, int32_t* fstate, int32_t flip_a, int32_t flip_b, double* tunes,
                             int sm_count, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  if (N < 2 || N > kMaxFftTurns || N > n_turn) return cudaErrorInvalidValue;
  const size_t smem = sizeof(double) * 4 * N;
  cudaError_t e = cudaSuccess;
  if (smem > 48 * 1024) e = cudaFuncSetAttribute(k_fma_tunes, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)sm_count * 8));
  k_fma_status<<<grid, 256, 0, s>>>(state, rec_state, n, fstate);
  k_fma_tunes<<<(unsigned)(n * 6), kTuneThreads, smem, s>>>(hist, n, n_turn, N, fstate, flip_a, flip_b, tunes);
  return cudaGetLastError();
}

}  // namespace bmadgpu

extern "C" int bmadgpu_fma(bmadgpu_ctx* c, const bmadgpu_lattice* lat, int32_t n_particles, const double* offsets,
                           const bmadgpu_fma_params* P, bmadgpu_fma_point* out) {
  if (!c || !lat || !P || !out || n_particles < 0 || (n_particles > 0 && !offsets)) return fail(BMADGPU_EINVAL, "bad argument");
  if (lat->device != c->device) return fail(BMADGPU_EINVAL, "lattice and context are on different devices");
  if (P->n_turn < 2) return fail(BMADGPU_EINVAL, "n_turn < 2");
  const int N = P->fft_turns > 0 ? P->fft_turns : P->n_turn / 2;
  if (N < 2 || N > P->n_turn) return fail(BMADGPU_EINVAL, "fft_turns must be in [2, n_turn]");
  if (N > kMaxFftTurns) return fail(BMADGPU_EINVAL, "fft_turns above 4096");
  if (n_particles == 0) return BMADGPU_OK;
  CUDA_TRY(cudaSetDevice(c->device));
  cudaStream_t s = c->stream;

  // z_cut: a quarter of the lowest RF wavelength of the cavities (frequency_map.f90:99-119).
  double z_limit = 0;
  if (P->z_cut) {
    double f = P->rf_frequency;
    if (f <= 0) {
      f = 0;
      for (const auto& e : lat->eles)
        if (e.key == BMADGPU_RFCAVITY) f = (f == 0) ? e.rf_frequency : std::fmin(f, e.rf_frequency);
    }
    if (f > 0) z_limit = 0.25 * (kCLight / f);
  }

  // particles per chunk: the turn-by-turn record (48 B per particle-turn) within 8 GiB
  const int64_t per = (int64_t)48 * P->n_turn;
  const int64_t chunk = std::max<int64_t>(1, std::min<int64_t>(n_particles, ((int64_t)8 << 30) / per));
  std::vector<void*> mem;
  struct Free {
    std::vector<void*>& m;
    ~Free() {
      for (void* p : m) cudaFree(p);
    }
  } freer{mem};
  auto get = [&](size_t bytes) -> void* {
    void* p = nullptr;
    if (cudaMalloc(&p, bytes) != cudaSuccess) return nullptr;
    mem.push_back(p);
    return p;
  };
  const int64_t m = chunk;
  double* hist = (double*)get(sizeof(double) * 6 * P->n_turn * m);
  double* d_off = (double*)get(sizeof(double) * 6 * m);
  double* d_par = (double*)get(sizeof(double) * 42);  // norm [36], co [6]
  double* d_tunes = (double*)get(sizeof(double) * 6 * m);
  bmadgpu_bunch b;
  b.n = m;
  b.vec = (double*)get(sizeof(double) * 6 * m);
  b.beta = (double*)get(sizeof(double) * m);
  b.t = nullptr;
  b.state = (int32_t*)get(sizeof(int32_t) * m);
  b.ix_ele = (int32_t*)get(sizeof(int32_t) * m);
  b.ix_turn = (int32_t*)get(sizeof(int32_t) * m);
  b.location = (int32_t*)get(sizeof(int32_t) * m);
  int32_t* fstate = (int32_t*)get(sizeof(int32_t) * 3 * m);
  if (!hist || !d_off || !d_par || !d_tunes || !b.vec || !b.beta || !b.state || !b.ix_ele || !b.ix_turn ||
      !b.location || !fstate)
    return fail(BMADGPU_ENOMEM, "cannot allocate the frequency-map record");
  int32_t* fturn = fstate + m;
  int32_t* fele = fstate + 2 * m;
  double par[42];
  std::memcpy(par, P->norm, sizeof(double) * 36);
  std::memcpy(par + 36, P->orbit, sizeof(double) * 6);
  CUDA_TRY(cudaMemcpyAsync(d_par, par, sizeof(par), cudaMemcpyHostToDevice, s));
  const int flip_a = P->tune_a < 0.5, flip_b = P->tune_b < 0.5;
  const size_t smem = sizeof(double) * 4 * N;
  if (smem > 48 * 1024) CUDA_TRY(cudaFuncSetAttribute(k_fma_tunes, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  std::vector<double> h_tunes;
  std::vector<int32_t> h_f;

  for (int64_t base = 0; base < n_particles; base += chunk) {
    const int64_t cn = std::min<int64_t>(chunk, n_particles - base);
    b.n = cn;
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((cn + 255) / 256, (int64_t)c->sm_count * 8));
    CUDA_TRY(cudaMemcpyAsync(d_off, offsets + base * 6, sizeof(double) * 6 * cn, cudaMemcpyHostToDevice, s));
    k_fma_start<<<grid, 256, 0, s>>>(d_off, d_par + 36, cn, lat->param.p0c, lat->param.e_tot, lat->param.mass, b.vec,
                                     b.beta, b.state, b.ix_ele, b.ix_turn, b.location, fstate);
    CUDA_TRY(cudaGetLastError());
    c->launches++;
    for (int32_t turn = 0; turn < P->n_turn; turn++) {
      int r = track_device(c, lat, &b, 0, (int32_t)lat->pk.info.n_ele, turn, 1, nullptr);
      if (r) return r;
      k_fma_record<<<grid, 256, 0, s>>>(b.vec, b.state, b.ix_ele, cn, turn, P->n_turn, d_par, d_par + 36, z_limit,
                                        hist, fstate, fturn, fele);
      CUDA_TRY(cudaGetLastError());
      c->launches++;
    }
    k_fma_tunes<<<(unsigned)(cn * 6), kTuneThreads, smem, s>>>(hist, cn, P->n_turn, N, fstate, flip_a, flip_b, d_tunes);
    CUDA_TRY(cudaGetLastError());
    c->launches++;
    h_tunes.resize(6 * cn);
    h_f.resize(3 * cn);
    CUDA_TRY(cudaMemcpyAsync(h_tunes.data(), d_tunes, sizeof(double) * 6 * cn, cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaMemcpyAsync(h_f.data(), fstate, sizeof(int32_t) * cn, cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaMemcpyAsync(h_f.data() + cn, fturn, sizeof(int32_t) * cn, cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaMemcpyAsync(h_f.data() + 2 * cn, fele, sizeof(int32_t) * cn, cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    for (int64_t i = 0; i < cn; i++) {
      bmadgpu_fma_point& o = out[base + i];
      std::memset(&o, 0, sizeof(o));
      o.status = h_f[i];
      if (o.status == 0) {
        for (int k = 0; k < 6; k++) o.tune[k] = h_tunes[i * 6 + k];
      } else {
        o.turn_lost = h_f[cn + i];
        o.ix_ele = o.status == 1 ? h_f[2 * cn + i] : -1;
      }
    }
  }
  return check_err_flag(c);
}

// The reference's .fm table (frequency_map.f90:236-242, 376-381): a '(12a14)' header, then per
// particle x, y, pz, the three first-half tunes, the three second-half tunes and their differences
// as '(12e14.5)', or the offsets as '(3e14.5)' and '*' in the nine tune columns.
namespace {

// Fortran Ew.d with d = 5: [-]0.ddddd E+ee (E dropped for three-digit exponents), right-justified.
void fmt_e14_5(char* buf, double v) {
  if (v == 0) {
    std::snprintf(buf, 15, "%14s", std::signbit(v) ? "-0.00000E+00" : "0.00000E+00");
    return;
  }
  char tmp[40];
  std::snprintf(tmp, sizeof(tmp), "%.4E", std::fabs(v));  // d.ddddE+xx: the 5 significant digits, rounded
  const char* e = std::strchr(tmp, 'E');
  const int ex = std::atoi(e + 1) + 1;                    // 0.ddddd x 10^ex
  char out[40];
  if (std::abs(ex) <= 99)
    std::snprintf(out, sizeof(out), "%s0.%c%c%c%c%cE%c%02d", v < 0 ? "-" : "", tmp[0], tmp[2], tmp[3], tmp[4], tmp[5],
                  ex < 0 ? '-' : '+', std::abs(ex));
  else
    std::snprintf(out, sizeof(out), "%s0.%c%c%c%c%c%c%03d", v < 0 ? "-" : "", tmp[0], tmp[2], tmp[3], tmp[4], tmp[5],
                  ex < 0 ? '-' : '+', std::abs(ex));
  const size_t len = std::min<size_t>(std::strlen(out), 14);
  std::memset(buf, ' ', 14 - len);
  std::memcpy(buf + 14 - len, out, len);
  buf[14] = 0;
}

}  // namespace

extern "C" int bmadgpu_fma_write(const char* path, int32_t n_particles, const double* offsets,
                                 const bmadgpu_fma_point* points, int32_t append) {
  if (!path || n_particles < 0 || (n_particles > 0 && (!offsets || !points))) return BMADGPU_EINVAL;
  FILE* f = std::fopen(path, append ? "a" : "w");
  if (!f) return BMADGPU_EINVAL;
  if (!append) {
    static const char* head[12] = {"# x", "y", "pz", "Qx0", "Qy0", "Qz0", "Qx1", "Qy1", "Qz1", "dQx", "dQy", "dQz"};
    for (int k = 0; k < 12; k++) std::fprintf(f, "%14s", head[k]);
    std::fprintf(f, "\n");
  }
  char b[16];
  for (int32_t i = 0; i < n_particles; i++) {
    const bmadgpu_fma_point& p = points[i];
    if (p.status == 1) continue;  // lost particles get no line (frequency_map.f90:326)
    const double* o = offsets + 6 * (int64_t)i;
    const double lead[3] = {o[0], o[2], o[5]};
    for (double v : lead) {
      fmt_e14_5(b, v);
      std::fputs(b, f);
    }
    if (p.status == 0) {
      for (int k = 0; k < 6; k++) {
        fmt_e14_5(b, p.tune[k]);
        std::fputs(b, f);
      }
      for (int k = 0; k < 3; k++) {
        fmt_e14_5(b, p.tune[3 + k] - p.tune[k]);
        std::fputs(b, f);
      }
    } else {
      for (int k = 0; k < 9; k++) std::fprintf(f, "%14s", "*");
    }
    std::fprintf(f, "\n");
  }
  return std::fclose(f) == 0 ? BMADGPU_OK : BMADGPU_EINVAL;
}
