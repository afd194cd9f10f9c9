// optics.cu -- closed orbit, one-turn matrix, periodic Twiss and the matched Gaussian beam: what
// long_term_tracking sets up before tracking (twiss_and_track, lt_tracking_mod.f90:562;
// ltt_init_beam_distribution, lt_tracking_mod.f90:1548-1561).
//
// Closed orbit (closed_orbit_calc, bmad/code/closed_orbit_calc.f90:192-862). The reference fits the
// fixed point of the one-turn map with super_mrqmin, taking the Jacobian from the analytic element
// matrices (make_mat6). Here the one-turn map is this library's own device tracking, and the
// Jacobian comes from it too: every Newton step tracks 25 particles for one turn in one launch --
// the trial orbit and x +- h e_k, x +- 2h e_k for each coordinate -- and the fourth-order central
// difference of those gives the one-turn matrix (h = 1e-5: truncation (h / A)^4 ~ 1e-12 for
// nonlinear scales A ~ 1 cm, rounding ~1e-13). The fixed point found is the reference's: it does
// not depend on how the Jacobian is had, only on the map and the stopping rule, which is the
// reference's (all |f(x)_i - x_i| < |x_i| rel_tol + abs_tol over the fitted coordinates).
//
// Periodic Twiss (twiss_at_start.f90:29 -> twiss_from_mat6.f90:24 -> mat_symp_decouple.f90:22,
// twiss_from_mat2.f90:19): the symplectic decoupling of the 4x4 transverse block into the a and b
// modes, Twiss of each, and the dispersion (I - M4)^-1 M(1:4, 6).
//
// Matched beam (init_bunch_distribution / init_random_distribution,
// bmad/multiparticle/beam_utils.f90:328-535, 551-721): standard normal deviates per particle, the
// finite-sample renormalisation (zero mean, unit covariance by the reference's sequence of shears),
// the Twiss/sigma scaling, the centroid renormalisation, dispersion and coupling (make_v_mats), the
// beam centre and the closed orbit (add_closed_orbit_to_init_position). The bulk is device kernels
// over the SoA bunch; the 6x6 covariance the shears need comes from the deterministic device sums
// of the bunch statistics (stats.cu) and the 15 shear factors are computed on the host as the
// reference computes them, then applied on the device in the reference's order.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "capi_internal.h"
#include "stats.cuh"

using namespace bmadgpu;

namespace {

constexpr double kCLight = 299792458.0;   // c_light (physical_constants.f90)
constexpr double kTwoPi = 6.283185307179586;
constexpr int kStencil = 25;              // the orbit, then x + h, x - h, x + 2h, x - 2h per coordinate
constexpr double kFdStep = 1e-5;

// ---- small dense linear algebra (row-major) -------------------------------------------------

// Solves A x = b in place (n <= 6) by Gaussian elimination with partial pivoting.
bool solve(int n, double* A, double* b) {
  for (int c = 0; c < n; c++) {
    int p = c;
    for (int r = c + 1; r < n; r++)
      if (std::fabs(A[r * n + c]) > std::fabs(A[p * n + c])) p = r;
    if (A[p * n + c] == 0) return false;
    if (p != c) {
      for (int k = 0; k < n; k++) std::swap(A[c * n + k], A[p * n + k]);
      std::swap(b[c], b[p]);
    }
    for (int r = c + 1; r < n; r++) {
      const double f = A[r * n + c] / A[c * n + c];
      for (int k = c; k < n; k++) A[r * n + k] -= f * A[c * n + k];
      b[r] -= f * b[c];
    }
  }
  for (int r = n - 1; r >= 0; r--) {
    double s = b[r];
    for (int k = r + 1; k < n; k++) s -= A[r * n + k] * b[k];
    b[r] = s / A[r * n + r];
  }
  return true;
}

// 2x2 symplectic conjugate [[d, -b], [-c, a]] (mat_symp_conj).
void conj2(const double* m, double* o) {
  o[0] = m[3];
  o[1] = -m[1];
  o[2] = -m[2];
  o[3] = m[0];
}

// 4x4 symplectic conjugate: conj([[A, B], [C, D]]) = [[conj A, conj C], [conj B, conj D]].
void conj4(const double* m, double* o) {
  for (int bi = 0; bi < 2; bi++)
    for (int bj = 0; bj < 2; bj++) {
      const double blk[4] = {m[(2 * bj) * 4 + 2 * bi], m[(2 * bj) * 4 + 2 * bi + 1], m[(2 * bj + 1) * 4 + 2 * bi],
                             m[(2 * bj + 1) * 4 + 2 * bi + 1]};
      double c[4];
      conj2(blk, c);
      o[(2 * bi) * 4 + 2 * bj] = c[0];
      o[(2 * bi) * 4 + 2 * bj + 1] = c[1];
      o[(2 * bi + 1) * 4 + 2 * bj] = c[2];
      o[(2 * bi + 1) * 4 + 2 * bj + 1] = c[3];
    }
}

void mul4(const double* a, const double* b, double* o) {
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) {
      double s = 0;
      for (int k = 0; k < 4; k++) s += a[i * 4 + k] * b[k * 4 + j];
      o[i * 4 + j] = s;
    }
}

// max |M^T S M - S| (mat_symp_error, sim_utils/matrix/mat_symp_error.f90).
double symp_error4(const double* m) {
  double err = 0;
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) {
      double s = 0;
      for (int p = 0; p < 2; p++)  // (M^T S M)_ij = sum_p M_{2p,i} M_{2p+1,j} - M_{2p+1,i} M_{2p,j}
        s += m[(2 * p) * 4 + i] * m[(2 * p + 1) * 4 + j] - m[(2 * p + 1) * 4 + i] * m[(2 * p) * 4 + j];
      const double sij = (i / 2 == j / 2) ? (i % 2 == 0 && j % 2 == 1 ? 1.0 : (i % 2 == 1 && j % 2 == 0 ? -1.0 : 0.0))
                                          : 0.0;
      err = std::fmax(err, std::fabs(s - sij));
    }
  return err;
}

// Twiss of a 2x2 one-turn block (twiss_from_mat2.f90:19-60). Returns 0 ok, else the status.
int twiss_from_mat2(const double* min, double* beta, double* alpha, double* gamma, double* phi) {
  const double det = min[0] * min[3] - min[1] * min[2];
  const double m[4] = {min[0] / det, min[1] / det, min[2] / det, min[3] / det};
  const double t_cos = (m[0] + m[3]) / 2.0;
  if (std::fabs(t_cos) >= 1.0) return BMADGPU_TWISS_UNSTABLE;
  const double t_sin = std::copysign(1.0, m[1]) * std::sqrt(1.0 - t_cos * t_cos);
  double ph = std::atan2(t_sin, t_cos);
  if (ph < 0) ph += kTwoPi;
  const double a = (m[0] - m[3]) / (2.0 * t_sin);
  const double radical = -(1 + a * a) * m[1] / m[2];
  if (radical <= 0) return BMADGPU_TWISS_NON_SYMPLECTIC;
  *phi = ph;
  *alpha = a;
  *beta = std::sqrt(radical);
  *gamma = (1 + a * a) / *beta;
  return 0;
}

// ---- device scratch for the orbit particles -------------------------------------------------

struct OrbitParticles {
  void* mem = nullptr;
  bmadgpu_bunch b{};
  std::vector<double> hv, hb;
  std::vector<int32_t> hs;
  ~OrbitParticles() {
    if (mem) cudaFree(mem);
  }
  int init() {
    const int n = kStencil;
    if (cudaMalloc(&mem, sizeof(double) * 7 * n + sizeof(int32_t) * n) != cudaSuccess)
      return fail(BMADGPU_ENOMEM, "cannot allocate the orbit particles");
    b.n = n;
    b.vec = (double*)mem;
    b.beta = b.vec + 6 * n;
    b.state = (int32_t*)(b.beta + n);
    hv.resize(6 * n);
    hb.resize(n);
    hs.resize(n);
    return BMADGPU_OK;
  }
};

struct TmpLattice {
  bmadgpu_lattice* lat = nullptr;
  ~TmpLattice() {
    if (lat) bmadgpu_lattice_destroy(lat);
  }
};

bool rf_is_on(const bmadgpu_lattice* lat) {
  for (const auto& e : lat->eles)
    if (e.key == BMADGPU_RFCAVITY && e.is_on && e.voltage != 0) return true;
  return false;
}

// The lattice the orbit searches track: apertures off (closed_orbit_calc.f90:268) and, for the
// RF-off calculations, every rfcavity switched off (set_on_off(rfcavity$, ..., off_and_save$),
// closed_orbit_calc.f90:301; twiss_at_start.f90 tracks the cavities as drifts).
int orbit_lattice(bmadgpu_ctx* c, const bmadgpu_lattice* lat, bool rf_off, TmpLattice& tmp) {
  bmadgpu_param p = lat->param;
  p.aperture_limit_on = 0;
  std::vector<bmadgpu_element> e = lat->eles;
  if (rf_off)
    for (auto& x : e)
      if (x.key == BMADGPU_RFCAVITY) x.is_on = 0;
  return bmadgpu_lattice_create(c, e.data(), (int32_t)e.size(), &p, &tmp.lat);
}

double init_beta(const bmadgpu_param& p, double pz) {
  if (pz == 0) return p.p0c / p.e_tot;
  const double pc = p.p0c * (1 + pz);
  return pc / std::sqrt(pc * pc + p.mass * p.mass);
}

// One turn of the 25 stencil particles about x: f(x) and the one-turn matrix. *lost is set when
// any of them is lost (the caller's cue to step back: the matrix needs all 25).
int one_turn(bmadgpu_ctx* c, const bmadgpu_lattice* lat, const double* x, double* fx, double* M,
             OrbitParticles& op, bool* lost) {
  const int n = kStencil;
  static const double kOff[4] = {1, -1, 2, -2};
  for (int j = 0; j < n; j++) {
    for (int i = 0; i < 6; i++) op.hv[i * n + j] = x[i];
    if (j > 0) op.hv[((j - 1) / 4) * n + j] += kOff[(j - 1) % 4] * kFdStep;
    op.hb[j] = init_beta(lat->param, op.hv[5 * n + j]);
    op.hs[j] = BMADGPU_ALIVE;
  }
  cudaStream_t s = c->stream;
  CUDA_TRY(cudaMemcpyAsync(op.b.vec, op.hv.data(), sizeof(double) * 6 * n, cudaMemcpyHostToDevice, s));
  CUDA_TRY(cudaMemcpyAsync(op.b.beta, op.hb.data(), sizeof(double) * n, cudaMemcpyHostToDevice, s));
  CUDA_TRY(cudaMemcpyAsync(op.b.state, op.hs.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice, s));
  int r = track_device(c, lat, &op.b, 0, (int32_t)lat->pk.info.n_ele, 0, 1, nullptr);
  if (r) return r;
  CUDA_TRY(cudaMemcpyAsync(op.hv.data(), op.b.vec, sizeof(double) * 6 * n, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaMemcpyAsync(op.hs.data(), op.b.state, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  if ((r = check_err_flag(c))) return r;
  *lost = false;
  for (int j = 0; j < n; j++) *lost = *lost || op.hs[j] != BMADGPU_ALIVE;
  if (*lost) return BMADGPU_OK;
  for (int i = 0; i < 6; i++) fx[i] = op.hv[i * n];
  for (int i = 0; i < 6; i++)
    for (int k = 0; k < 6; k++) {
      const double* row = &op.hv[i * n + 1 + 4 * k];
      M[i * 6 + k] = (8 * (row[0] - row[1]) - (row[2] - row[3])) / (12 * kFdStep);
    }
  return BMADGPU_OK;
}

// Largest |eigenvalue| of the longitudinal 2x2 block: the z-mode stability test of max_z_eigen
// (closed_orbit_calc.f90:755-766), taken on the block instead of the full 6x6 eigen-decomposition
// (the same verdict when synchro-betatron coupling is weak). A complex pair is stable and counts
// as 1; a real pair gives its larger modulus.
double z_eigen(const double* M) {
  const double a = M[4 * 6 + 4], b = M[4 * 6 + 5], c = M[5 * 6 + 4], d = M[5 * 6 + 5];
  const double h = 0.5 * (a + d), det = a * d - b * c, disc = h * h - det;
  if (disc < 0) return 1.0;
  const double s = std::sqrt(disc);
  return std::fmax(std::fabs(h + s), std::fabs(h - s));
}

// ---- matched beam kernels -------------------------------------------------------------------

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC11):
// ten rounds of two 32x32->64 multiplies with the published multipliers and Weyl key increments.
__host__ __device__ inline void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
  for (int r = 0; r < 10; r++) {
    const uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
    const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    c[0] = hi1 ^ c[1] ^ k0;
    c[1] = lo1;
    c[2] = hi0 ^ c[3] ^ k1;
    c[3] = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
}

// Standard normal deviate number k of stream index i (Box-Muller on two 53-bit uniforms in (0, 1));
// with cut > 0 the deviate is redrawn (next attempt counter) until |r| <= cut, as ran_gauss does
// with a sigma cutoff (random_mod.f90:172-394), at most 64 times.
__device__ double gauss_deviate(uint64_t seed, uint64_t i, uint32_t k, double cut) {
  for (uint32_t a = 0; a < 64; a++) {
    uint32_t c[4] = {(uint32_t)i, (uint32_t)(i >> 32), a, k};
    philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    const double u1 = ((double)((((uint64_t)c[0]) << 21) | (c[1] >> 11)) + 0.5) * 0x1p-53;
    const double u2 = ((double)((((uint64_t)c[2]) << 21) | (c[3] >> 11)) + 0.5) * 0x1p-53;
    const double r = sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
    if (cut <= 0 || fabs(r) <= cut) return r;
  }
  return 0.0;
}

// vec [6][n] gets the particle deviates; extra [8] the two sigma jitters and six centre jitters
// (stream indices n and n + 1).
__global__ void k_gauss(double* __restrict__ vec, int64_t n, double* __restrict__ extra, uint64_t seed, double cut) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
    for (int k = 0; k < 6; k++) vec[k * n + i] = gauss_deviate(seed, (uint64_t)i, k, cut);
  if (blockIdx.x == 0 && threadIdx.x < 8) {
    const int t = threadIdx.x;
    extra[t] = gauss_deviate(seed, (uint64_t)n + (t < 2 ? 0 : 1), t < 2 ? t : t - 2, cut);
  }
}

__global__ void k_set_alive(int32_t* __restrict__ state, int64_t n) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) state[i] = BMADGPU_ALIVE;
}

struct ShapeArgs {
  int32_t renorm, n_ops, scale, pad;
  int32_t oi[15], oj[15];
  double ob[15];
  double ave[6], alpha[6];
  double sigma[6];
  double alpha_a, alpha_b, a, b;
};

// Renormalisation and Twiss/sigma scaling (beam_utils.f90:604-699).
__global__ void k_shape(double* __restrict__ vec, int64_t n, ShapeArgs A) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    double r[6];
    for (int k = 0; k < 6; k++) r[k] = vec[k * n + i];
    if (A.renorm) {
      for (int k = 0; k < 6; k++) r[k] = r[k] - A.ave[k];
      for (int o = 0; o < A.n_ops; o++) r[A.oi[o]] = r[A.oi[o]] + A.ob[o] * r[A.oj[o]];
      if (A.scale)
        for (int k = 0; k < 6; k++) r[k] = r[k] * A.alpha[k];
    }
    vec[0 * n + i] = A.sigma[0] * r[0];
    vec[1 * n + i] = -A.sigma[1] * (r[1] + r[0] * A.alpha_a);
    vec[2 * n + i] = A.sigma[2] * r[2];
    vec[3 * n + i] = -A.sigma[3] * (r[3] + r[2] * A.alpha_b);
    vec[4 * n + i] = A.sigma[4] * r[4];
    vec[5 * n + i] = A.sigma[5] * (r[5] * A.b + r[4] * A.a);
  }
}

struct FinishArgs {
  int32_t recenter, pad;
  double ave[6];
  double eta[4];      // a%eta, a%etap, b%eta, b%etap
  double v[16];       // v_mat (make_v_mats), row-major
  double offset[6];   // beam centre (+ jitter)
  double orbit[6];    // closed orbit, or zero
  double p0c, e_tot, mass;
};

// Centroid renormalisation, dispersion and coupling, centre and closed orbit, then the particle
// set-up of init_coord (beam_utils.f90:702-711, 491-509, 1920-1923; lt_tracking_mod.f90:1555-1559;
// init_coord.f90:205-222).
__global__ void k_finish(double* __restrict__ vec, double* __restrict__ beta, double* __restrict__ t,
                         int32_t* __restrict__ state, int32_t* __restrict__ ix_ele, int32_t* __restrict__ ix_turn,
                         int32_t* __restrict__ location, int64_t n, FinishArgs F) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    double r[6];
    for (int k = 0; k < 6; k++) r[k] = vec[k * n + i];
    if (F.recenter)
      for (int k = 0; k < 6; k++) r[k] = r[k] - F.ave[k];
    double pt[4];
    for (int k = 0; k < 4; k++) pt[k] = r[k] + r[5] * F.eta[k];
    for (int k = 0; k < 4; k++)
      r[k] = F.v[k * 4 + 0] * pt[0] + F.v[k * 4 + 1] * pt[1] + F.v[k * 4 + 2] * pt[2] + F.v[k * 4 + 3] * pt[3];
    for (int k = 0; k < 6; k++) r[k] = r[k] + F.offset[k];
    for (int k = 0; k < 6; k++) r[k] = r[k] + F.orbit[k];
    for (int k = 0; k < 6; k++) vec[k * n + i] = r[k];
    double b;
    if (r[5] == 0) {
      b = F.p0c / F.e_tot;
    } else {
      const double pc = F.p0c * (1 + r[5]);
      b = pc / sqrt(pc * pc + F.mass * F.mass);
    }
    beta[i] = b;
    if (t) t[i] = -r[4] / (b * kCLight);
    state[i] = BMADGPU_ALIVE;
    if (ix_ele) ix_ele[i] = -1;
    if (ix_turn) ix_turn[i] = -1;
    if (location) location[i] = 0;
  }
}

int grid_for(const bmadgpu_ctx* c, int64_t n) {
  const int64_t want = (n + 255) / 256;
  const int64_t cap = (int64_t)c->sm_count * 8;
  return (int)std::max<int64_t>(1, std::min(want, cap));
}

}  // namespace

// ---- closed orbit ----------------------------------------------------------------------------

extern "C" int bmadgpu_one_turn_matrix(bmadgpu_ctx* c, const bmadgpu_lattice* lat, const double* orbit,
                                       int32_t rf_on, double* orbit_end, double* mat) {
  if (!c || !lat || !orbit || !mat) return fail(BMADGPU_EINVAL, "NULL argument");
  if (lat->device != c->device) return fail(BMADGPU_EINVAL, "lattice and context are on different devices");
  CUDA_TRY(cudaSetDevice(c->device));
  TmpLattice tmp;
  int r = orbit_lattice(c, lat, !rf_on, tmp);
  if (r) return r;
  OrbitParticles op;
  if ((r = op.init())) return r;
  double fx[6];
  bool lost = false;
  if ((r = one_turn(c, tmp.lat, orbit, fx, mat, op, &lost))) return r;
  if (lost) return fail(BMADGPU_EINVAL, "the orbit particle or one of its stencil neighbours was lost in one turn");
  if (orbit_end) std::memcpy(orbit_end, fx, sizeof(fx));
  return BMADGPU_OK;
}

extern "C" int bmadgpu_closed_orbit(bmadgpu_ctx* c, const bmadgpu_lattice* lat, int32_t dim, double* orbit,
                                    double* mat, double rel_tol, double abs_tol, int32_t max_iter,
                                    int32_t* iterations) {
  if (!c || !lat || !orbit) return fail(BMADGPU_EINVAL, "NULL argument");
  if (lat->device != c->device) return fail(BMADGPU_EINVAL, "lattice and context are on different devices");
  const bool rf_on = rf_is_on(lat);
  if (dim == 0) dim = rf_on ? 6 : 4;
  if (dim != 4 && dim != 5 && dim != 6) return fail(BMADGPU_EINVAL, "dim must be 4, 5 or 6");
  if (dim == 6 && !rf_on) return fail(BMADGPU_EINVAL, "cannot do the 6-dimensional closed orbit with no RF voltage");
  if (rel_tol <= 0) rel_tol = 1e-9;   // bmad_com%rel_tol_tracking (bmad_struct.f90:2318)
  if (abs_tol <= 0) abs_tol = 1e-12;  // bmad_com%abs_tol_tracking (bmad_struct.f90:2319)
  if (max_iter <= 0) max_iter = 100;  // i_max (closed_orbit_calc.f90:390)
  CUDA_TRY(cudaSetDevice(c->device));
  TmpLattice tmp;
  int r = orbit_lattice(c, lat, dim != 6, tmp);
  if (r) return r;
  OrbitParticles op;
  if ((r = op.init())) return r;

  // RF wavelength for the z step limit and the z window (closed_orbit_calc.f90:318-327, 523).
  double rf_freq = 1e30;
  for (const auto& e : lat->eles)
    if (e.key == BMADGPU_RFCAVITY && e.is_on) rf_freq = std::fmin(rf_freq, std::fabs(e.rf_frequency));
  const double rf_wavelen = kCLight * (lat->param.p0c / lat->param.e_tot) / rf_freq;

  // Unknowns: x, px, y, py (+ z for dim 6); dim 5 fits pz in place of z so that z returns.
  const int nu = dim;
  int ix[6] = {0, 1, 2, 3, 4, 5};
  if (dim == 5) ix[4] = 5;
  double x[6];
  for (int i = 0; i < 6; i++) x[i] = orbit[i];
  if (dim != 6) x[4] = 0;  // start_orb%vec(5) = 0 (closed_orbit_calc.f90:311)

  double fx[6], M[36], last_step[6] = {0, 0, 0, 0, 0, 0};
  bool alive_once = false, tried_zero = false, z_checked = false, converged = false;
  int halvings = 0, it = 0;
  for (; it < max_iter; ++it) {
    bool lost = false;
    if ((r = one_turn(c, tmp.lat, x, fx, M, op, &lost))) return r;
    if (lost) {
      if (alive_once && halvings < 30) {  // the last step overshot: take half of it
        for (int i = 0; i < nu; i++) {
          last_step[i] *= 0.5;
          x[ix[i]] -= last_step[i];
        }
        ++halvings;
        continue;
      }
      if (!alive_once && !tried_zero) {  // "desperation move" (closed_orbit_calc.f90:420-425)
        for (int i = 0; i < std::min(5, nu); i++) x[ix[i]] = 0;
        tried_zero = true;
        continue;
      }
      return fail(BMADGPU_EINVAL, "particle lost in tracking: aborting the closed-orbit search");
    }
    alive_once = true;
    halvings = 0;
    // Residual on the fitted coordinates: x, px, y, py, z (dims 5 and 6), not pz (closed_orbit_calc.f90:65-73).
    double res[6];
    bool ok = true;
    for (int i = 0; i < nu; i++) {
      res[i] = fx[i] - x[i];
      if (!(std::fabs(res[i]) < std::fabs(x[i]) * rel_tol + abs_tol)) ok = false;
    }
    if (ok) {
      if (dim == 6 && z_eigen(M) >= 1.000001 && !z_checked) {
        // Unstable longitudinal fixed point: scan z in steps of lambda/8 (closed_orbit_calc.f90:622-645).
        z_checked = true;
        const double z0 = x[4];
        double best = z_eigen(M), best_z = z0;
        for (int j = -3; j <= 4; j++) {
          if (j == 0) continue;
          double xs[6], fs[6], Ms[36];
          std::memcpy(xs, x, sizeof(xs));
          xs[4] = z0 + j * rf_wavelen / 8;
          bool l2 = false;
          if ((r = one_turn(c, tmp.lat, xs, fs, Ms, op, &l2))) return r;
          if (l2) continue;
          const double e = z_eigen(Ms);
          if (e < best) {
            best = e;
            best_z = xs[4];
          }
        }
        x[4] = best_z;
        continue;
      }
      converged = true;
      break;
    }
    // Newton step: (M - I) dx = -(f(x) - x) on the unknowns (dim 5: column pz, co_func's dy_da).
    double A[36], b[6];
    for (int i = 0; i < nu; i++) {
      for (int k = 0; k < nu; k++) A[i * nu + k] = M[i * 6 + ix[k]] - (ix[k] == i ? 1.0 : 0.0);
      b[i] = -res[i];
    }
    if (!solve(nu, A, b)) return fail(BMADGPU_EINVAL, "one-turn matrix minus the identity is singular");
    if (dim == 6) {  // limit the z step to lambda_rf / 10 (closed_orbit_calc.f90:48-57)
      const double dz_norm = std::fabs(b[4]) / (rf_wavelen / 10);
      if (dz_norm > 1)
        for (int i = 0; i < nu; i++) b[i] /= dz_norm;
    }
    for (int i = 0; i < nu; i++) {
      x[ix[i]] += b[i];
      last_step[i] = b[i];
    }
    if (dim == 6) {  // keep z within half a wavelength (modulo2, closed_orbit_calc.f90:523)
      const double h = rf_wavelen / 2;
      x[4] = x[4] - 2 * h * std::floor((x[4] + h) / (2 * h));
    }
  }
  if (iterations) *iterations = it;
  if (!converged) return fail(BMADGPU_ETIMEDOUT, "closed orbit not converging");
  for (int i = 0; i < 6; i++) orbit[i] = x[i];
  if (mat) std::memcpy(mat, M, sizeof(M));
  return BMADGPU_OK;
}

// ---- periodic Twiss --------------------------------------------------------------------------

extern "C" int bmadgpu_twiss_from_mat6(const double* mat6, const double* orb0, bmadgpu_twiss* tw) {
  if (!mat6 || !tw) return BMADGPU_EINVAL;
  std::memset(tw, 0, sizeof(*tw));
  tw->gamma_c = 1;
  double m4[16];
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) m4[i * 4 + j] = mat6[i * 6 + j];
  double mx = 0;
  for (double v : m4) mx = std::fmax(mx, std::fabs(v));
  if (mx > 1e10) {  // twiss_from_mat6.f90:63-70
    tw->status = BMADGPU_TWISS_UNSTABLE;
    tw->growth_rate = mx;
    return BMADGPU_OK;
  }
  const double se = symp_error4(m4);
  tw->symp_error = se;
  if (se > 1) {
    tw->status = BMADGPU_TWISS_NON_SYMPLECTIC;
    tw->growth_rate = std::fmin(1e5 * se, mx);
    return BMADGPU_OK;
  }

  // mat_symp_decouple (mat_symp_decouple.f90:56-104): V = [[g I, C], [-conj C, g I]], U = conj(V) M V.
  double gamma = 1, C[4] = {0, 0, 0, 0};
  const double Mm[4] = {m4[0], m4[1], m4[4], m4[5]}, mm[4] = {m4[2], m4[3], m4[6], m4[7]};
  const double nn[4] = {m4[8], m4[9], m4[12], m4[13]}, Nn[4] = {m4[10], m4[11], m4[14], m4[15]};
  if (!(mm[0] == 0 && mm[1] == 0 && mm[2] == 0 && mm[3] == 0)) {
    double nc[4], H[4];
    conj2(nn, nc);
    for (int k = 0; k < 4; k++) H[k] = mm[k] + nc[k];
    const double tdiff = (Mm[0] + Mm[3]) - (Nn[0] + Nn[3]);
    const double det_h = H[0] * H[3] - H[1] * H[2];
    const double denom = tdiff * tdiff + 4.0 * det_h;
    if (denom <= 0) {
      tw->status = BMADGPU_TWISS_IN_STOP_BAND;
      tw->growth_rate = std::sqrt(std::fmax(std::fabs(2 * (1 - denom)) - 2, 0.0));
      return BMADGPU_OK;
    }
    gamma = std::sqrt(0.5 + 0.5 * std::sqrt(tdiff * tdiff / denom));
    const double scalar = -std::copysign(1.0, tdiff) / (gamma * std::sqrt(denom));
    for (int k = 0; k < 4; k++) C[k] = scalar * H[k];
  }
  double V[16] = {0}, Vc[16], U[16], T[16];
  for (int i = 0; i < 4; i++) V[i * 4 + i] = gamma;
  double cc[4];
  conj2(C, cc);
  V[0 * 4 + 2] = C[0];
  V[0 * 4 + 3] = C[1];
  V[1 * 4 + 2] = C[2];
  V[1 * 4 + 3] = C[3];
  V[2 * 4 + 0] = -cc[0];
  V[2 * 4 + 1] = -cc[1];
  V[3 * 4 + 0] = -cc[2];
  V[3 * 4 + 1] = -cc[3];
  conj4(V, Vc);
  mul4(Vc, m4, T);
  mul4(T, V, U);
  const double tra = U[0] + U[5], trb = U[10] + U[15];
  if (std::fabs(tra) > 2 || std::fabs(trb) > 2) {
    tw->status = (std::fabs(tra) > 2 && std::fabs(trb) > 2) ? BMADGPU_TWISS_UNSTABLE
                 : (std::fabs(tra) > 2)                    ? BMADGPU_TWISS_UNSTABLE_A
                                                           : BMADGPU_TWISS_UNSTABLE_B;
    const double r1 = std::sqrt(std::fmax(std::fabs(tra) - 2, 0.0)), r2 = std::sqrt(std::fmax(std::fabs(trb) - 2, 0.0));
    tw->growth_rate = std::fmax(r1, r2);
    if (tw->growth_rate > 1e4) tw->growth_rate = 1e4 + 1e2 * std::log10(tw->growth_rate - 1e4 + 1.0);
    return BMADGPU_OK;
  }
  const double Ua[4] = {U[0], U[1], U[4], U[5]}, Ub[4] = {U[10], U[11], U[14], U[15]};
  if (twiss_from_mat2(Ua, &tw->beta_a, &tw->alpha_a, &tw->gamma_a, &tw->phi_a)) {
    tw->status = BMADGPU_TWISS_UNSTABLE_A;
    return BMADGPU_OK;
  }
  if (twiss_from_mat2(Ub, &tw->beta_b, &tw->alpha_b, &tw->gamma_b, &tw->phi_b)) {
    tw->status = BMADGPU_TWISS_UNSTABLE_B;
    return BMADGPU_OK;
  }
  tw->gamma_c = gamma;
  for (int k = 0; k < 4; k++) tw->c_mat[k] = C[k];

  // Dispersion (twiss_from_mat6.f90:96-124): eta = (I - M4)^-1 M(1:4, 6); normal modes conj(V) eta.
  double A[16], e[4];
  for (int i = 0; i < 4; i++) {
    for (int j = 0; j < 4; j++) A[i * 4 + j] = (i == j ? 1.0 : 0.0) - m4[i * 4 + j];
    e[i] = mat6[i * 6 + 5];
  }
  if (solve(4, A, e)) {
    tw->eta_x = e[0];
    tw->etap_x = e[1];
    tw->eta_y = e[2];
    tw->etap_y = e[3];
    double en[4];
    for (int i = 0; i < 4; i++) en[i] = Vc[i * 4 + 0] * e[0] + Vc[i * 4 + 1] * e[1] + Vc[i * 4 + 2] * e[2] + Vc[i * 4 + 3] * e[3];
    tw->eta_a = en[0];
    tw->etap_a = en[1];
    tw->eta_b = en[2];
    tw->etap_b = en[3];
  }
  // deta_ds as twiss_from_mat6.f90:104-124 writes them (the y and b terms divide by rel_p and
  // multiply by 2 as written there).
  const double rel_p = 1 + (orb0 ? orb0[5] : 0.0);
  const double o[4] = {orb0 ? orb0[0] : 0.0, orb0 ? orb0[1] : 0.0, orb0 ? orb0[2] : 0.0, orb0 ? orb0[3] : 0.0};
  tw->deta_ds_x = tw->etap_x / rel_p - o[1] / (rel_p * rel_p);
  tw->deta_ds_y = tw->etap_y / rel_p - o[3] / rel_p * 2;
  double vo[4];
  for (int i = 0; i < 4; i++) vo[i] = Vc[i * 4 + 0] * o[0] + Vc[i * 4 + 1] * o[1] + Vc[i * 4 + 2] * o[2] + Vc[i * 4 + 3] * o[3];
  tw->deta_ds_a = tw->etap_a / rel_p - vo[1] / (rel_p * rel_p);
  tw->deta_ds_b = tw->etap_b / rel_p - vo[3] / rel_p * 2;
  tw->status = BMADGPU_TWISS_OK;
  return BMADGPU_OK;
}

// ---- matched Gaussian beam -------------------------------------------------------------------

extern "C" int bmadgpu_beam_init_gaussian(bmadgpu_ctx* c, const bmadgpu_param* param, const bmadgpu_twiss* tw,
                                          const bmadgpu_beam_init* bi, const double* normals, const double* orbit,
                                          bmadgpu_bunch* b) {
  if (!c || !param || !tw || !bi || !b || !b->vec || !b->beta || !b->state) return fail(BMADGPU_EINVAL, "NULL argument");
  const int64_t n = b->n;
  if (n < 1) return fail(BMADGPU_EINVAL, "number of particles to init for beam is zero");
  if (tw->beta_a <= 0 || tw->beta_b <= 0) return fail(BMADGPU_EINVAL, "Twiss beta must be positive");
  CUDA_TRY(cudaSetDevice(c->device));
  cudaStream_t s = c->stream;
  const int grid = grid_for(c, n);

  // scratch: deviates of the jitters, statistics partials and sums
  void* mem = nullptr;
  const size_t scratch = sizeof(double) * (8 + (size_t)kStatBlocks * kStatPass2 + kStatSums);
  if (cudaMalloc(&mem, scratch) != cudaSuccess) return fail(BMADGPU_ENOMEM, "cannot allocate the beam-init scratch");
  struct Free {
    void* p;
    ~Free() { cudaFree(p); }
  } freer{mem};
  double* d_extra = (double*)mem;
  double* d_partial = d_extra + 8;
  double* d_sums = d_partial + (size_t)kStatBlocks * kStatPass2;

  double extra[8];
  if (normals) {
    CUDA_TRY(cudaMemcpyAsync(b->vec, normals, sizeof(double) * 6 * n, cudaMemcpyDeviceToDevice, s));
    CUDA_TRY(cudaMemcpyAsync(d_extra, normals + 6 * n, sizeof(double) * 8, cudaMemcpyDeviceToDevice, s));
  } else {
    k_gauss<<<grid, 256, 0, s>>>(b->vec, n, d_extra, bi->seed, bi->sigma_cutoff);
    CUDA_TRY(cudaGetLastError());
    c->launches++;
  }
  k_set_alive<<<grid, 256, 0, s>>>(b->state, n);
  CUDA_TRY(cudaGetLastError());
  c->launches++;
  CUDA_TRY(cudaMemcpyAsync(extra, d_extra, sizeof(extra), cudaMemcpyDeviceToHost, s));

  ShapeArgs A;
  std::memset(&A, 0, sizeof(A));
  if (bi->renorm_sigma) {
    // ave and sig_mat of the deviates (beam_utils.f90:588-597), from the device sums.
    CUDA_TRY(launch_bunch_sums(b->vec, nullptr, b->state, n, d_partial, d_sums, s));
    c->launches += 4;
    double sums[kStatSums];
    CUDA_TRY(cudaMemcpyAsync(sums, d_sums, sizeof(sums), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    double ave[6], sig[36];
    for (int i = 0; i < 6; i++) ave[i] = sums[1 + i] / n;
    for (int i = 0, q = 9; i < 6; i++)
      for (int j = i; j < 6; j++, q++) sig[i * 6 + j] = sig[j * 6 + i] = sums[q] / n;
    // renorm_sigma (beam_utils.f90:608-651): zero mean, shears that zero the off-diagonal
    // covariance in the reference's order, then unit diagonal.
    A.renorm = 1;
    for (int i = 0; i < 6; i++) A.ave[i] = ave[i];
    for (int i = 0; i < 6; i++)
      for (int j = 0; j < 6; j++) sig[i * 6 + j] = sig[i * 6 + j] - ave[i] * ave[j];
    if (n > 6) {
      for (int i = 4; i >= 0; i--)
        for (int j = i + 1; j < 6; j++) {
          const double bb = -sig[i * 6 + j] / sig[j * 6 + j];
          A.oi[A.n_ops] = i;
          A.oj[A.n_ops] = j;
          A.ob[A.n_ops] = bb;
          A.n_ops++;
          sig[i * 6 + i] = sig[i * 6 + i] + 2 * bb * sig[i * 6 + j] + bb * bb * sig[j * 6 + j];
          for (int j2 = 0; j2 < 6; j2++) {
            if (j2 == i) continue;
            sig[i * 6 + j2] = sig[i * 6 + j2] + bb * sig[j * 6 + j2];
            sig[j2 * 6 + i] = sig[i * 6 + j2];
          }
        }
    }
    if (n > 1) {
      A.scale = 1;
      for (int i = 0; i < 6; i++) A.alpha[i] = std::sqrt(1 / sig[i * 6 + i]);
    }
  } else {
    CUDA_TRY(cudaStreamSynchronize(s));
  }
  // sigmas (beam_utils.f90:662-693)
  A.sigma[0] = std::sqrt(bi->a_emit * tw->beta_a);
  A.sigma[1] = std::sqrt(bi->a_emit / tw->beta_a);
  A.sigma[2] = std::sqrt(bi->b_emit * tw->beta_b);
  A.sigma[3] = std::sqrt(bi->b_emit / tw->beta_b);
  A.sigma[4] = bi->sig_z * (1 + bi->sig_z_jitter * extra[0]);
  A.sigma[5] = bi->sig_pz * (1 + bi->sig_pz_jitter * extra[1]);
  if (A.sigma[5] == 0 || bi->dpz_dz == 0) {
    A.a = 0;
  } else if (std::fabs(bi->dpz_dz * A.sigma[4]) > A.sigma[5]) {
    return fail(BMADGPU_EINVAL, "|dpz_dz| must be < sig_pz / sig_z");
  } else {
    A.a = bi->dpz_dz * A.sigma[4] / A.sigma[5];
  }
  A.b = std::sqrt(1 - A.a * A.a);
  A.alpha_a = tw->alpha_a;
  A.alpha_b = tw->alpha_b;
  k_shape<<<grid, 256, 0, s>>>(b->vec, n, A);
  CUDA_TRY(cudaGetLastError());
  c->launches++;

  FinishArgs F;
  std::memset(&F, 0, sizeof(F));
  if (bi->renorm_center) {  // beam_utils.f90:702-711
    CUDA_TRY(launch_bunch_sums(b->vec, nullptr, b->state, n, d_partial, d_sums, s));
    c->launches += 4;
    double sums[kStatSums];
    CUDA_TRY(cudaMemcpyAsync(sums, d_sums, sizeof(sums), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    F.recenter = 1;
    for (int i = 0; i < 6; i++) F.ave[i] = sums[1 + i] / n;
  }
  F.eta[0] = tw->eta_a;
  F.eta[1] = tw->etap_a;
  F.eta[2] = tw->eta_b;
  F.eta[3] = tw->etap_b;
  // v_mat (make_v_mats.f90:33-38)
  double cc[4];
  conj2(tw->c_mat, cc);
  const double g = tw->gamma_c;
  const double v[16] = {g, 0, tw->c_mat[0], tw->c_mat[1], 0, g, tw->c_mat[2], tw->c_mat[3],
                        -cc[0], -cc[1], g, 0, -cc[2], -cc[3], 0, g};
  std::memcpy(F.v, v, sizeof(v));
  for (int k = 0; k < 6; k++) F.offset[k] = bi->center[k] + bi->center_jitter[k] * extra[2 + k];
  if (orbit)
    for (int k = 0; k < 6; k++) F.orbit[k] = orbit[k];
  F.p0c = param->p0c;
  F.e_tot = param->e_tot;
  F.mass = param->mass;
  k_finish<<<grid, 256, 0, s>>>(b->vec, b->beta, b->t, b->state, b->ix_ele, b->ix_turn, b->location, n, F);
  CUDA_TRY(cudaGetLastError());
  c->launches++;
  CUDA_TRY(cudaStreamSynchronize(s));
  return BMADGPU_OK;
}

extern "C" int bmadgpu_gaussian_deviates(bmadgpu_ctx* c, uint64_t seed, double sigma_cutoff, int64_t n, double* d_out) {
  if (!c || !d_out || n < 0) return fail(BMADGPU_EINVAL, "bad argument");
  if (n == 0) return BMADGPU_OK;
  CUDA_TRY(cudaSetDevice(c->device));
  void* mem = nullptr;
  if (cudaMalloc(&mem, sizeof(double) * 8) != cudaSuccess) return fail(BMADGPU_ENOMEM, "cannot allocate");
  k_gauss<<<grid_for(c, n), 256, 0, c->stream>>>(d_out, n, (double*)mem, seed, sigma_cutoff);
  cudaError_t e = cudaGetLastError();
  c->launches++;
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_out + 6 * n, mem, sizeof(double) * 8, cudaMemcpyDeviceToDevice, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  cudaFree(mem);
  if (e != cudaSuccess) return cuda_fail(e, "bmadgpu_gaussian_deviates");
  return BMADGPU_OK;
}

extern "C" int bmadgpu_philox4x32_10(const uint32_t* counter, const uint32_t* key, uint32_t* out) {
  if (!counter || !key || !out) return BMADGPU_EINVAL;
  uint32_t c[4] = {counter[0], counter[1], counter[2], counter[3]};
  philox4x32_10(c, key[0], key[1]);
  for (int i = 0; i < 4; i++) out[i] = c[i];
  return BMADGPU_OK;
}
