// ltt.cu -- the long-term-tracking beam-mode driver: turn loop, stop conditions and the averages
// and phase-space outputs of ltt_run_beam_mode (bsim/modules/lt_tracking_mod.f90:1571-1715),
// ltt_write_averages_data (:2613-2713, headers :758-846) and ltt_write_particle_data
// (:1904-2057), over a device-resident bunch.
//
// Tracking runs in chunks between output turns (one k_track launch per chunk, live-list
// compaction inside long chunks). The stop conditions of the turn loop -- no particle left, or
// the lost count reaching nint(dead_cutoff * n) -- are checked on the per-turn live counts the
// kernel reduces; if one fires inside a chunk, the chunk is re-run from a copy of its starting
// state for exactly the turns up to the stopping turn, so the bunch ends where the reference's
// loop exits and no output is written for that turn, as there.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <utility>
#include <vector>

#include "capi_internal.h"
#include "stats.cuh"

using namespace bmadgpu;

namespace {

// Fortran ESw.d: d digits after the point, exponent E+dd, or +ddd without the E (3-digit).
std::string fmt_es(int w, int d, double x) {
  char buf[64];
  std::snprintf(buf, sizeof buf, "%.*E", d, x);
  std::string s(buf);
  size_t e = s.find('E');
  if (e != std::string::npos) {
    std::string mant = s.substr(0, e), ex = s.substr(e + 1);
    int ev = std::atoi(ex.c_str());
    char eb[16];
    if (std::abs(ev) < 100) std::snprintf(eb, sizeof eb, "E%c%02d", ev < 0 ? '-' : '+', std::abs(ev));
    else std::snprintf(eb, sizeof eb, "%c%03d", ev < 0 ? '-' : '+', std::abs(ev));
    s = mant + eb;
  }
  if ((int)s.size() < w) s = std::string(w - s.size(), ' ') + s;
  if ((int)s.size() > w) s = std::string(w, '*');
  return s;
}

std::string fmt_f(int w, int d, double x) {
  char buf[64];
  std::snprintf(buf, sizeof buf, "%*.*f", w, d, x);
  std::string s(buf);
  if ((int)s.size() > w) s = std::string(w, '*');
  return s;
}

std::string fmt_i(int w, long long v) {
  char buf[32];
  std::snprintf(buf, sizeof buf, "%*lld", w, v);
  return buf;
}

const char* state_name(int st) {  // coord_state_name, bmad/modules/bmad_struct.f90:2635-2659
  switch (st) {
    case 1: return "Alive";
    case 2: return "Lost";
    case 3: return "Lost_Neg_X";
    case 4: return "Lost_Pos_X";
    case 5: return "Lost_Neg_Y";
    case 6: return "Lost_Pos_Y";
    case 7: return "Lost_Z";
    case 8: return "Lost_Pz";
    case -999: return "Not_Set";
    default: return "null";
  }
}

// Output schedule of ltt_write_averages_data / ltt_write_particle_data.
bool wants(int every, int only_last, int n_turns, int turn) {
  if (every > 0 && only_last > 0 && n_turns - turn >= only_last) return false;
  if (every == -1) return turn == n_turns;
  if (every == 0) return turn == 0 || turn == n_turns;
  if (every < 0) return false;
  return turn % every == 0;
}

struct DevBunch {
  std::vector<void*> ptrs;
  bmadgpu_bunch b;
  bool alloc(int64_t n) {
    std::memset(&b, 0, sizeof(b));
    b.n = n;
    void* p;
    auto get = [&](size_t bytes) -> void* {
      if (cudaMalloc(&p, bytes + 16) != cudaSuccess) return nullptr;
      ptrs.push_back(p);
      return p;
    };
    b.vec = (double*)get(6 * n * sizeof(double));
    b.beta = (double*)get(n * sizeof(double));
    b.t = (double*)get(n * sizeof(double));
    b.state = (int32_t*)get(n * sizeof(int32_t));
    b.ix_ele = (int32_t*)get(n * sizeof(int32_t));
    b.ix_turn = (int32_t*)get(n * sizeof(int32_t));
    b.location = (int32_t*)get(n * sizeof(int32_t));
    return b.vec && b.beta && b.t && b.state && b.ix_ele && b.ix_turn && b.location;
  }
  ~DevBunch() {
    for (void* p : ptrs) cudaFree(p);
  }
};

cudaError_t copy_bunch(const bmadgpu_bunch& dst, const bmadgpu_bunch& src, cudaMemcpyKind kind, cudaStream_t s,
                       bool with_t, bool with_loss) {
  const size_t nd = (size_t)src.n * sizeof(double), ni = (size_t)src.n * sizeof(int32_t);
  cudaError_t e;
  if ((e = cudaMemcpyAsync(dst.vec, src.vec, 6 * nd, kind, s)) != cudaSuccess) return e;
  if ((e = cudaMemcpyAsync(dst.beta, src.beta, nd, kind, s)) != cudaSuccess) return e;
  if ((e = cudaMemcpyAsync(dst.state, src.state, ni, kind, s)) != cudaSuccess) return e;
  if (with_t && (e = cudaMemcpyAsync(dst.t, src.t, nd, kind, s)) != cudaSuccess) return e;
  if (with_loss) {
    if ((e = cudaMemcpyAsync(dst.ix_ele, src.ix_ele, ni, kind, s)) != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(dst.ix_turn, src.ix_turn, ni, kind, s)) != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(dst.location, src.location, ni, kind, s)) != cudaSuccess) return e;
  }
  return cudaSuccess;
}

std::string preheader(const bmadgpu_lattice* lat, const bmadgpu_ltt_params* P) {
  char buf[512];
  std::string h;
  const double t0 = lat->pk.ref_time_prefix.back();
  std::snprintf(buf, sizeof buf, "# e_tot                                     = %s\n", fmt_es(0, 6, lat->param.e_tot).c_str());
  h += buf;
  std::snprintf(buf, sizeof buf, "# t_1turn                                   = %s\n", fmt_es(0, 6, t0).c_str());
  h += buf;
  std::snprintf(buf, sizeof buf, "# ltt%%tracking_method                       = \"BMAD\"\n");
  h += buf;
  std::snprintf(buf, sizeof buf, "# ltt%%n_turns                               = %d\n", P->n_turns);
  h += buf;
  std::snprintf(buf, sizeof buf, "# ltt%%averages_output_every_n_turns         = %d\n", P->averages_every_n_turns);
  h += buf;
  std::snprintf(buf, sizeof buf, "# ltt%%particle_output_every_n_turns         = %d\n", P->particle_every_n_turns);
  h += buf;
  return h;
}

std::string col(int w, const char* s) {
  std::string x(s);
  if ((int)x.size() < w) x = std::string(w - x.size(), ' ') + x;
  return x;
}

bool write_averages_headers(const std::string& base, const std::string& pre, const double* cuts, int n_cuts) {
  FILE* f = std::fopen((base + ".ave").c_str(), "w");
  if (!f) return false;
  std::string l1 = "##" + col(8, "1") + col(9, "2") + col(14, "3") + col(14, "4");
  std::string l2 = "##" + col(8, "Turn") + col(9, "N_live") + col(14, "Time") + col(14, "Polarization");
  const char* a3[] = {"<Sx>", "<Sy>", "<Sz>"};
  for (int i = 0; i < 3; i++) {
    l1 += col(14, std::to_string(5 + i).c_str());
    l2 += col(14, a3[i]);
  }
  l1 += "  ";
  l2 += "  ";
  const char* a8[] = {"<x>", "<px>", "<y>", "<py>", "<z>", "<pz>", "<pc>", "<p0c>"};
  for (int i = 0; i < 8; i++) {
    l1 += col(14, std::to_string(8 + i).c_str());
    l2 += col(14, a8[i]);
  }
  l1 += "  ";
  l2 += "  ";
  const char* a6[] = {"Sig_x", "Sig_px", "Sig_y", "Sig_py", "Sig_z", "Sig_pz"};
  for (int i = 0; i < 6; i++) {
    l1 += col(14, std::to_string(16 + i).c_str());
    l2 += col(14, a6[i]);
  }
  std::fprintf(f, "%s%s\n%s\n", pre.c_str(), l1.c_str(), l2.c_str());
  std::fclose(f);

  f = std::fopen((base + ".sigma").c_str(), "w");
  if (!f) return false;
  l1 = "##" + col(8, "1") + col(9, "2") + col(12, "3") + "  ";
  l2 = "##" + col(8, "Turn") + col(9, "N_live") + col(12, "Time") + "  ";
  const char* names[] = {"x", "px", "y", "py", "z", "pz"};
  int k = 0;
  for (int i = 0; i < 6; i++)
    for (int j = i; j < 6; j++, k++) {
      l1 += col(14, std::to_string(4 + k).c_str());
      l2 += col(14, ("<" + std::string(names[i]) + "." + names[j] + ">").c_str());
    }
  std::fprintf(f, "%s%s\n%s\n", pre.c_str(), l1.c_str(), l2.c_str());
  std::fclose(f);

  f = std::fopen((base + ".emit").c_str(), "w");
  if (!f) return false;
  l1 = "##" + col(8, "1") + col(10, "2") + col(12, "3") + "  ";
  l2 = "##" + col(8, "Turn") + col(10, "N_live") + col(12, "Time") + "  ";
  const char* e9[] = {"Emit_a", "Emit_b", "Emit_c", "Kurtosis_x", "Kurtosis_y", "Kurtosis_z", "Skew_x", "Skew_y", "Skew_z"};
  for (int i = 0; i < 9; i++) {
    l1 += col(14, std::to_string(4 + i).c_str());
    l2 += col(14, e9[i]);
    if (i == 2 || i == 5) {
      l1 += "  ";
      l2 += "  ";
    }
  }
  l1 += "  |";
  l2 += "  |";
  for (int i = 0; i < n_cuts; i++) {  // lt_tracking_mod.f90:832-839
    l1 += "                   " + std::to_string((int)std::lround(cuts[i] * 100)) + "% Core                |";
    l2 += "      Emit_a        Emit_b        Emit_c   |";
  }
  std::fprintf(f, "%s%s\n%s\n", pre.c_str(), l1.c_str(), l2.c_str());
  std::fclose(f);
  return true;
}

bool append_averages(const std::string& base, int turn, const bmadgpu_bunch_data& bd, const double* core, int n_cuts) {
  const std::string t_str = fmt_i(10, turn);
  FILE* f = std::fopen((base + ".ave").c_str(), "a");
  if (!f) return false;
  std::string l = t_str + fmt_i(9, bd.n_live) + fmt_es(14, 6, bd.t) + fmt_f(14, 9, 0.0) + "  ";
  for (int i = 0; i < 3; i++) l += fmt_f(14, 9, 0.0);   // spin is not tracked
  l += "  ";
  for (int i = 0; i < 6; i++) l += fmt_es(14, 6, bd.centroid[i]);
  l += fmt_es(14, 6, (1.0 + bd.centroid[5]) * bd.p0c) + fmt_es(14, 6, bd.p0c) + "  ";
  for (int i = 0; i < 6; i++) l += fmt_es(14, 6, bd.sig1[i]);
  std::fprintf(f, "%s\n", l.c_str());
  std::fclose(f);

  f = std::fopen((base + ".sigma").c_str(), "a");
  if (!f) return false;
  l = t_str + fmt_i(9, bd.n_live) + fmt_es(14, 6, bd.t) + "  ";
  for (int k = 0; k < 21; k++) l += fmt_es(14, 6, bd.sigma_vec[k]);
  std::fprintf(f, "%s\n", l.c_str());
  std::fclose(f);

  f = std::fopen((base + ".emit").c_str(), "a");
  if (!f) return false;
  l = t_str + fmt_i(9, bd.n_live) + fmt_es(14, 6, bd.t) + "  ";
  for (int i = 0; i < 3; i++) l += fmt_es(14, 6, bd.emit[i]);
  l += "  ";
  for (int i = 0; i < 3; i++) l += fmt_es(14, 6, bd.kurt[i]);
  l += "  ";
  for (int i = 0; i < 3; i++) l += fmt_es(14, 6, bd.skew[i]);
  for (int k = 0; k < n_cuts; k++) {
    l += "  ";
    for (int i = 0; i < 3; i++) l += fmt_es(14, 6, core[k * 3 + i]);
  }
  std::fprintf(f, "%s\n", l.c_str());
  std::fclose(f);
  return true;
}

// File name of write_this_data (lt_tracking_mod.f90:1972-1986): the turn zero-padded to the digits
// of n_turns replaces a '#' in the base name, or is appended.
std::string particle_file_name(const std::string& base, int turn, int n_turns) {
  std::string num;
  if (n_turns > 0) {
    const int width = (int)(std::log10((double)n_turns) + 1 + 1e-10);
    char b[32];
    std::snprintf(b, sizeof b, "%0*d", width, turn);
    num = b;
  } else {
    num = "000";
  }
  size_t ix = base.find('#');
  return ix == std::string::npos ? base + num : base.substr(0, ix) + num + base.substr(ix + 1);
}

bool write_phase_space(const std::string& base, int turn, int n_turns, const bmadgpu_bunch& h, double p0c,
                       bool only_live, const std::string& pre) {
  const std::string name = particle_file_name(base, turn, n_turns);
  FILE* f = std::fopen(name.c_str(), "w");
  if (!f) return false;
  std::fprintf(f, "%s", pre.c_str());
  std::fprintf(f, "##     Ix     Turn |           x              px               y              py               z "
                  "             pz              pc             p0c            time   |        spin_x       spin_y  "
                  "     spin_z    State\n");
  const int64_t n = h.n;
  for (int64_t j = 0; j < n; j++) {
    if (only_live && h.state[j] != 1) continue;
    std::string l = fmt_i(9, j + 1) + fmt_i(9, turn);
    for (int i = 0; i < 6; i++) l += fmt_es(16, 8, h.vec[i * n + j]);
    l += fmt_es(16, 8, (1.0 + h.vec[5 * n + j]) * p0c) + fmt_es(16, 8, p0c) + fmt_es(16, 8, h.t ? h.t[j] : 0.0);
    l += "   " + fmt_f(13, 9, 0.0) + fmt_f(13, 9, 0.0) + fmt_f(13, 9, 0.0) + "    " + state_name(h.state[j]);
    std::fprintf(f, "%s\n", l.c_str());
  }
  std::fclose(f);
  return true;
}

// Action-angle file of write_this_data (lt_tracking_mod.f90:1995-2049): per particle
// J_k = (j_2k^2 + j_2k+1^2) / 2 and angle_k = atan2(j_2k+1, j_2k), j = N^-1 (p - centroid), as the
// device computed them into aa [6][n].
bool write_action_angle(const std::string& base, int turn, int n_turns, const double* aa, const int32_t* state,
                        int64_t n, bool only_live, const std::string& pre) {
  const std::string name = particle_file_name(base, turn, n_turns);
  FILE* f = std::fopen(name.c_str(), "w");
  if (!f) return false;
  std::fprintf(f, "%s", pre.c_str());
  std::fprintf(f, "##     Ix     Turn |          Ja         Angle_a              Jb         Angle_b              Jc "
                  "        Angle_c   |     spin_x    spin_y    spin_z    State\n");
  for (int64_t j = 0; j < n; j++) {
    if (only_live && state[j] != 1) continue;
    std::string l = fmt_i(9, j + 1) + fmt_i(9, turn);
    for (int i = 0; i < 6; i++) l += fmt_es(16, 8, aa[i * n + j]);
    l += "   " + fmt_f(13, 9, 0.0) + fmt_f(13, 9, 0.0) + fmt_f(13, 9, 0.0) + "    " + state_name(state[j]);
    std::fprintf(f, "%s\n", l.c_str());
  }
  std::fclose(f);
  return true;
}

// ltt_per_particle_file_name (lt_tracking_mod.f90:725-752): the particle index zero-padded to
// int(log10(1.001 n_particle)) + 1 digits (a default-real product) replaces a '#', or follows a '.'.
std::string per_particle_file_name(const std::string& base, int64_t ip, int64_t n_particle) {
  const int np = (int)std::log10(1.001f * (float)n_particle) + 1;
  char b[32];
  std::snprintf(b, sizeof b, "%0*lld", np, (long long)ip);
  size_t ih = base.find('#');
  return ih == std::string::npos ? base + "." + b : base.substr(0, ih) + b + base.substr(ih + 1);
}

// ltt_write_per_particle_file_header (lt_tracking_mod.f90:690-720): one file per particle.
bool write_per_particle_headers(const std::string& base, int64_t n, const std::string& pre) {
  for (int64_t ip = 1; ip <= n; ip++) {
    FILE* f = std::fopen(per_particle_file_name(base, ip, n).c_str(), "w");
    if (!f) return false;
    std::fprintf(f, "%s# ix_bunch        = 1\n# ix_particle     = %lld\n", pre.c_str(), (long long)ip);
    std::fprintf(f, "##   Turn |           x              px               y              py               z          "
                    "    pz              pc             p0c            time   |    spin_x      spin_y      spin_z     "
                    "State\n");
    std::fclose(f);
  }
  return true;
}

// ltt_per_particle_file_write1 (lt_tracking_mod.f90:2062-2077): one line per particle and output turn.
bool append_per_particle(const std::string& base, int turn, const bmadgpu_bunch& h, double p0c) {
  const int64_t n = h.n;
  for (int64_t j = 0; j < n; j++) {
    FILE* f = std::fopen(per_particle_file_name(base, j + 1, n).c_str(), "a");
    if (!f) return false;
    std::string l = fmt_i(9, turn);
    for (int i = 0; i < 6; i++) l += fmt_es(16, 8, h.vec[i * n + j]);
    l += fmt_es(16, 8, (1.0 + h.vec[5 * n + j]) * p0c) + fmt_es(16, 8, p0c) + fmt_es(16, 8, h.t ? h.t[j] : 0.0);
    l += " " + fmt_f(12, 8, 0.0) + fmt_f(12, 8, 0.0) + fmt_f(12, 8, 0.0) + "    " + state_name(h.state[j]);
    std::fprintf(f, "%s\n", l.c_str());
    std::fclose(f);
  }
  return true;
}

// ---- core emittance (ltt_calc_bunch_data, lt_tracking_mod.f90:2432-2560) ----
//
// The reference ranks the live particles by their combined normalised amplitude
// sum_k (j_2k^2 + j_2k+1^2) / emit_k with j = N^-1 (p - centroid), N the normal-form matrix of the
// bunch's sigma matrix (Sigma = N diag(emit) N^T), keeps the n_cut = int(cutoff n_live) smallest,
// repeats the ranking with the core's own centroid and sigma, and scales that core's normal-mode
// emittances by f = cutoff / (1 - (1 + s + s^2/2 + s^3/6) e^-s), where e^-s solves
// ltt_beam_fraction(e^-s) = cutoff. Since Sigma^-1 = N^-T diag(1/emit) N^-1, the amplitude is the
// quadratic form (p - c)^T Sigma^-1 (p - c) = |L^-1 (p - c)|^2 with Sigma = L L^T: the device
// evaluates that per particle and selects the core (select_core), and the core's sums are the same
// two-pass device sums as the bunch's, over the core as the live set.
//
// With core_emit_combined_calc off (:2496-2516) each mode k has its own core: the particles of
// smallest action (j_2k^2 + j_2k+1^2) / 2 with N^-1 of the bunch, then of the core, and
// f = cutoff / (1 - (1 + s) e^-s), s = -ln(1 - cutoff).

constexpr int kCoreMax = 8;

struct CoreArgs {
  double w[36];    // row-major: L^-1 (combined) or N^-1 (one mode)
  double wgt[6];   // amplitude = sum_r wgt_r (w (p - c))_r^2
  double c[6];
};

__global__ void k_core_amp(const double* __restrict__ vec, const int32_t* __restrict__ state, int64_t n, CoreArgs A,
                           double* __restrict__ amp) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    if (state[i] != BMADGPU_ALIVE) {
      amp[i] = 1e100;  // the reference's "something large" for dead particles
      continue;
    }
    double d[6];
    for (int k = 0; k < 6; k++) d[k] = vec[k * n + i] - A.c[k];
    double s = 0;
    for (int r = 0; r < 6; r++) {
      if (A.wgt[r] == 0) continue;
      double y = 0;
      for (int k = 0; k < 6; k++) y += A.w[r * 6 + k] * d[k];
      s += A.wgt[r] * (y * y);
    }
    amp[i] = s;
  }
}

// Action and angle of every particle (dead ones too, as the reference writes them):
// aa [6][n] = J_a, angle_a, J_b, angle_b, J_c, angle_c with j = w (p - c).
__global__ void k_action_angle(const double* __restrict__ vec, int64_t n, CoreArgs A, double* __restrict__ aa) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    double d[6], j[6];
    for (int k = 0; k < 6; k++) d[k] = vec[k * n + i] - A.c[k];
    for (int r = 0; r < 6; r++) {
      double y = 0;
      for (int k = 0; k < 6; k++) y += A.w[r * 6 + k] * d[k];
      j[r] = y;
    }
    for (int m = 0; m < 3; m++) {
      aa[(2 * m) * n + i] = 0.5 * (j[2 * m] * j[2 * m] + j[2 * m + 1] * j[2 * m + 1]);
      aa[(2 * m + 1) * n + i] = atan2(j[2 * m + 1], j[2 * m]);
    }
  }
}

// Inverse of a 6x6 matrix by Gauss-Jordan elimination with partial pivoting (mat_inverse,
// sim_utils/matrix/mat_inverse.f90:19-56, uses LAPACK's getrf/getri); false if singular.
bool mat_inverse6(const double* a_in, double* inv) {
  double a[36];
  for (int i = 0; i < 36; i++) {
    a[i] = a_in[i];
    inv[i] = (i % 7 == 0) ? 1.0 : 0.0;
  }
  for (int col = 0; col < 6; col++) {
    int piv = col;
    for (int r = col + 1; r < 6; r++)
      if (std::fabs(a[r * 6 + col]) > std::fabs(a[piv * 6 + col])) piv = r;
    if (a[piv * 6 + col] == 0) return false;
    if (piv != col)
      for (int k = 0; k < 6; k++) {
        std::swap(a[piv * 6 + k], a[col * 6 + k]);
        std::swap(inv[piv * 6 + k], inv[col * 6 + k]);
      }
    const double p = a[col * 6 + col];
    for (int k = 0; k < 6; k++) {
      a[col * 6 + k] /= p;
      inv[col * 6 + k] /= p;
    }
    for (int r = 0; r < 6; r++) {
      if (r == col) continue;
      const double f = a[r * 6 + col];
      if (f == 0) continue;
      for (int k = 0; k < 6; k++) {
        a[r * 6 + k] -= f * a[col * 6 + k];
        inv[r * 6 + k] -= f * inv[col * 6 + k];
      }
    }
  }
  return true;
}

// N^-1 of a bunch's sigma matrix (calc_bunch_params' n_mat, then mat_inverse); false where the
// reference's eigen-analysis fails.
bool normal_form_inverse(const bmadgpu_bunch_data& bd, double* n_inv) {
  double n_mat[36];
  if (bd.n_live < 6 || !bd.emit_valid) return false;
  if (bmadgpu_sigma_normal_form(bd.sigma, nullptr, n_mat) != BMADGPU_OK) return false;
  return mat_inverse6(n_mat, n_inv);
}

// L^-1 of sigma = L L^T (6x6), false unless sigma is positive definite.
bool chol_inverse(const double* sig, double* li) {
  double L[36] = {0}, Li[36] = {0};
  for (int j = 0; j < 6; j++) {
    double s = sig[j * 6 + j];
    for (int k = 0; k < j; k++) s -= L[j * 6 + k] * L[j * 6 + k];
    if (!(s > 0)) return false;
    L[j * 6 + j] = std::sqrt(s);
    for (int i = j + 1; i < 6; i++) {
      double t = sig[i * 6 + j];
      for (int k = 0; k < j; k++) t -= L[i * 6 + k] * L[j * 6 + k];
      L[i * 6 + j] = t / L[j * 6 + j];
    }
  }
  for (int j = 0; j < 6; j++) {  // forward substitution column by column
    Li[j * 6 + j] = 1 / L[j * 6 + j];
    for (int i = j + 1; i < 6; i++) {
      double t = 0;
      for (int k = j; k < i; k++) t += L[i * 6 + k] * Li[k * 6 + j];
      Li[i * 6 + j] = -t / L[i * 6 + i];
    }
  }
  int q = 0;
  for (int r = 0; r < 6; r++)
    for (int k = 0; k <= r; k++) li[q++] = Li[r * 6 + k];
  return true;
}

// ltt_beam_fraction (lt_tracking_mod.f90:2566-2570): the share of a Gaussian beam inside the
// combined normalised amplitude -ln(x).
double beam_fraction(double x) {
  const double jc = -std::log(x);
  return 1.0 - x * (1 + jc + 0.5 * jc * jc);
}

// Brent's root finder (R. P. Brent, Algorithms for Minimization without Derivatives, 1973, ch. 4)
// for beam_fraction(x) = y on [a, b], run to full precision (the reference's inverse() stops at
// 1e-8; the root it approaches is this one).
double fraction_root(double y, double a, double b) {
  double fa = beam_fraction(a) - y, fb = beam_fraction(b) - y;
  if (fa * fb > 0) return b;
  double c = a, fc = fa, d = b - a, e = d;
  for (int it = 0; it < 200; it++) {
    if ((fb > 0) == (fc > 0)) {
      c = a;
      fc = fa;
      d = e = b - a;
    }
    if (std::fabs(fc) < std::fabs(fb)) {
      a = b;
      b = c;
      c = a;
      fa = fb;
      fb = fc;
      fc = fa;
    }
    const double tol = 2 * 2.220446049250313e-16 * std::fabs(b) + 1e-300;
    const double m = 0.5 * (c - b);
    if (std::fabs(m) <= tol || fb == 0) return b;
    if (std::fabs(e) >= tol && std::fabs(fa) > std::fabs(fb)) {
      double p, q, r;
      const double sr = fb / fa;
      if (a == c) {
        p = 2 * m * sr;
        q = 1 - sr;
      } else {
        q = fa / fc;
        r = fb / fc;
        p = sr * (2 * m * q * (q - r) - (b - a) * (r - 1));
        q = (q - 1) * (r - 1) * (sr - 1);
      }
      if (p > 0) q = -q;
      p = std::fabs(p);
      if (2 * p < std::fmin(3 * m * q - std::fabs(tol * q), std::fabs(e * q))) {
        e = d;
        d = p / q;
      } else {
        d = m;
        e = m;
      }
    } else {
      d = m;
      e = m;
    }
    a = b;
    fa = fb;
    b += std::fabs(d) > tol ? d : (m > 0 ? tol : -tol);
    fb = beam_fraction(b) - y;
  }
  return b;
}

struct CoreScratch {
  double* d_amp = nullptr;
  int32_t* d_mask = nullptr;
  int32_t* d_eq = nullptr;            // indices of the particles whose amplitude ties the threshold
  unsigned int* d_count = nullptr;    // [256] histogram, then [1] count of ties
  std::vector<int32_t> eq;
  ~CoreScratch() {
    cudaFree(d_amp);
    cudaFree(d_mask);
    cudaFree(d_eq);
    cudaFree(d_count);
  }
  bool alloc(int64_t n) {
    if (d_amp) return true;
    return cudaMalloc(&d_amp, (size_t)n * sizeof(double)) == cudaSuccess &&
           cudaMalloc(&d_mask, (size_t)n * sizeof(int32_t)) == cudaSuccess &&
           cudaMalloc(&d_eq, (size_t)n * sizeof(int32_t)) == cudaSuccess &&
           cudaMalloc(&d_count, 256 * sizeof(unsigned int)) == cudaSuccess;
  }
};

// Selection of the n_cut smallest amplitudes on the device, ties going to the lower particle
// index (the order of a stable sort of the amplitudes). Amplitudes are non-negative, so their
// IEEE bit patterns order as unsigned integers: eight 8-bit radix passes find the n_cut-th key T
// exactly (a histogram of the keys that share the prefix found so far, per pass).
__global__ void k_select_hist(const double* __restrict__ amp, int64_t n, unsigned long long prefix,
                              unsigned long long prefix_mask, int shift, unsigned int* __restrict__ hist) {
  __shared__ unsigned int h[256];
  for (int i = threadIdx.x; i < 256; i += blockDim.x) h[i] = 0;
  __syncthreads();
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const unsigned long long k = (unsigned long long)__double_as_longlong(amp[i]);
    if ((k & prefix_mask) == prefix) atomicAdd(&h[(k >> shift) & 255ull], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 256; i += blockDim.x)
    if (h[i]) atomicAdd(&hist[i], h[i]);
}

// mask = keys below T, plus every key equal to T when all ties are taken; otherwise the tied
// indices are listed in eq for the host to take the lowest.
__global__ void k_select_mask(const double* __restrict__ amp, int64_t n, unsigned long long t, int take_all_ties,
                              int32_t* __restrict__ mask, int32_t* __restrict__ eq, unsigned int* __restrict__ n_eq) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const unsigned long long k = (unsigned long long)__double_as_longlong(amp[i]);
    int32_t m = k < t ? BMADGPU_ALIVE : 0;
    if (k == t) {
      if (take_all_ties) m = BMADGPU_ALIVE;
      else eq[atomicAdd(n_eq, 1u)] = (int32_t)i;
    }
    mask[i] = m;
  }
}

__global__ void k_select_ties(const int32_t* __restrict__ idx, int64_t count, int32_t* __restrict__ mask) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < count; k += stride) mask[idx[k]] = BMADGPU_ALIVE;
}

// The core mask in cs.d_mask; *ok false if the core would need a dead particle.
int select_core(bmadgpu_ctx* c, int64_t n, int64_t n_cut, CoreScratch& cs, bool* ok) {
  *ok = false;
  cudaStream_t s = c->stream;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)c->sm_count * 4));
  unsigned long long prefix = 0, pmask = 0;
  int64_t rank = n_cut;       // 1-based rank of the wanted key among those sharing the prefix
  unsigned int hist[256];
  unsigned int ties = 0;
  for (int pass = 0; pass < 8; pass++) {
    const int shift = 56 - 8 * pass;
    CUDA_TRY(cudaMemsetAsync(cs.d_count, 0, 256 * sizeof(unsigned int), s));
    k_select_hist<<<grid, 256, 0, s>>>(cs.d_amp, n, prefix, pmask, shift, cs.d_count);
    CUDA_TRY(cudaGetLastError());
    c->launches++;
    CUDA_TRY(cudaMemcpyAsync(hist, cs.d_count, sizeof(hist), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    int64_t cum = 0;
    int b = 0;
    for (; b < 255; b++) {
      if (cum + (int64_t)hist[b] >= rank) break;
      cum += hist[b];
    }
    rank -= cum;
    ties = hist[b];
    prefix |= (unsigned long long)b << shift;
    pmask |= 255ull << shift;
  }
  // the n_cut-th smallest is a dead particle's 1e100 (or an infinite or NaN amplitude, whose bits
  // order above it): fewer live particles of finite amplitude than n_cut
  if (prefix >= (unsigned long long)__builtin_bit_cast(unsigned long long, 1e99)) return BMADGPU_OK;
  const int take_all = (int64_t)ties == rank;
  CUDA_TRY(cudaMemsetAsync(cs.d_count, 0, sizeof(unsigned int), s));
  k_select_mask<<<grid, 256, 0, s>>>(cs.d_amp, n, prefix, take_all, cs.d_mask, cs.d_eq, cs.d_count);
  CUDA_TRY(cudaGetLastError());
  c->launches++;
  if (!take_all) {
    // a tie split by the cut: the lowest indices of the tied particles
    unsigned int n_eq = 0;
    CUDA_TRY(cudaMemcpyAsync(&n_eq, cs.d_count, sizeof(n_eq), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    cs.eq.resize(n_eq);
    CUDA_TRY(cudaMemcpyAsync(cs.eq.data(), cs.d_eq, n_eq * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    std::sort(cs.eq.begin(), cs.eq.end());
    const int64_t take = std::min<int64_t>(rank, (int64_t)n_eq);
    CUDA_TRY(cudaMemcpyAsync(cs.d_eq, cs.eq.data(), take * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    const int g2 = (int)std::max<int64_t>(1, std::min<int64_t>((take + 255) / 256, (int64_t)c->sm_count * 4));
    k_select_ties<<<g2, 256, 0, s>>>(cs.d_eq, take, cs.d_mask);
    CUDA_TRY(cudaGetLastError());
    c->launches++;
    CUDA_TRY(cudaStreamSynchronize(s));
  }
  *ok = true;
  return BMADGPU_OK;
}

// One ranking: the n_cut live particles of smallest amplitude about (centroid, sigma) of `ref` --
// the combined amplitude (mode 0) or the action of mode 1..3 -- and the bunch data of that core
// from the device sums.
int core_pass(bmadgpu_ctx* c, const bmadgpu_lattice* lat, const bmadgpu_bunch& d, double* d_scratch,
              const bmadgpu_bunch_data& ref, int mode, int64_t n_cut, CoreScratch& cs, bmadgpu_bunch_data* core,
              bool* ok) {
  *ok = false;
  CoreArgs A;
  for (int k = 0; k < 6; k++) A.wgt[k] = 0;
  if (mode == 0) {
    double li[21];
    if (!chol_inverse(ref.sigma, li)) return BMADGPU_OK;
    int q = 0;
    for (int r = 0; r < 6; r++)
      for (int k = 0; k < 6; k++) A.w[r * 6 + k] = k <= r ? li[q++] : 0.0;
    for (int k = 0; k < 6; k++) A.wgt[k] = 1;
  } else {
    if (!normal_form_inverse(ref, A.w)) return BMADGPU_OK;
    A.wgt[2 * mode - 2] = A.wgt[2 * mode - 1] = 0.5;
  }
  for (int k = 0; k < 6; k++) A.c[k] = ref.centroid[k];
  const int64_t n = d.n;
  cudaStream_t s = c->stream;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)c->sm_count * 8));
  k_core_amp<<<grid, 256, 0, s>>>(d.vec, d.state, n, A, cs.d_amp);
  CUDA_TRY(cudaGetLastError());
  c->launches++;
  // the n_cut smallest amplitudes, ties in particle order, selected on the device
  bool selected = false;
  int rs = select_core(c, n, n_cut, cs, &selected);
  if (rs || !selected) return rs;
  double sums[kStatSums];
  CUDA_TRY(launch_bunch_sums(d.vec, d.t, cs.d_mask, n, d_scratch, d_scratch + kStatBlocks * kStatPass2, s));
  c->launches += 4;
  CUDA_TRY(cudaMemcpyAsync(sums, d_scratch + kStatBlocks * kStatPass2, sizeof(sums), cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  int r = bmadgpu_bunch_data_from_sums(sums, lat->param.p0c, lat->param.mass, core);
  if (r) return r;
  *ok = core->emit_valid != 0;
  return BMADGPU_OK;
}

// core_emit [3] of one cutoff (zeros where the reference leaves them zero; with the per-mode
// calculation the modes before a failed one keep their values, as this_core_calc returns there).
int core_emittance(bmadgpu_ctx* c, const bmadgpu_lattice* lat, const bmadgpu_bunch& d, double* d_scratch,
                   const bmadgpu_bunch_data& bd, double cutoff_in, bool combined, CoreScratch& cs, double* out) {
  out[0] = out[1] = out[2] = 0;
  if (bd.n_live < 10) return BMADGPU_OK;
  if (!bd.emit_valid || bd.emit[0] == 0 || bd.emit[1] == 0 || bd.emit[2] == 0) return BMADGPU_OK;
  const int64_t n_cut = (int64_t)(cutoff_in * (double)bd.n_live);
  if (n_cut <= 0) return BMADGPU_OK;
  if (!cs.alloc(d.n)) return fail(BMADGPU_ENOMEM, "cannot allocate the core-emittance scratch");
  const double cutoff = std::fmin(1.0 - 1e-8, cutoff_in);
  bmadgpu_bunch_data core1, core2;
  bool ok = false;
  int r;
  if (combined) {
    const double sig_cut = -std::log(fraction_root(cutoff, 1e-12, 1.0));
    const double f =
        cutoff / (1 - (1 + sig_cut + sig_cut * sig_cut / 2 + sig_cut * sig_cut * sig_cut / 6) * std::exp(-sig_cut));
    r = core_pass(c, lat, d, d_scratch, bd, 0, n_cut, cs, &core1, &ok);
    if (r || !ok) return r;
    r = core_pass(c, lat, d, d_scratch, core1, 0, n_cut, cs, &core2, &ok);
    if (r || !ok) return r;
    for (int k = 0; k < 3; k++) out[k] = f * core2.emit[k];
    return BMADGPU_OK;
  }
  const double sig_cut = -std::log(1 - cutoff);
  const double f = cutoff / (1 - (1 + sig_cut) * std::exp(-sig_cut));
  for (int m = 1; m <= 3; m++) {
    r = core_pass(c, lat, d, d_scratch, bd, m, n_cut, cs, &core1, &ok);
    if (r || !ok) return r;
    r = core_pass(c, lat, d, d_scratch, core1, m, n_cut, cs, &core2, &ok);
    if (r || !ok) return r;
    out[m - 1] = f * core2.emit[m - 1];
  }
  return BMADGPU_OK;
}

// Action and angle of every particle of a device bunch into the host arrays aa [6][n]: about the
// bunch's own normal form and centroid (zero where the reference's eigen-analysis fails), or, with
// n_inv given (the one-turn matrix's N^-1), about zero.
int action_angle(bmadgpu_ctx* c, const bmadgpu_bunch& d, const bmadgpu_bunch_data& bd, const double* n_inv,
                 double* d_aa, double* aa) {
  CoreArgs A;
  if (n_inv) {
    for (int k = 0; k < 36; k++) A.w[k] = n_inv[k];
  } else if (!normal_form_inverse(bd, A.w)) {
    for (int k = 0; k < 36; k++) A.w[k] = 0;
  }
  for (int k = 0; k < 6; k++) {
    A.c[k] = (!n_inv && bd.n_live > 0) ? bd.centroid[k] : 0.0;
    A.wgt[k] = 0;
  }
  const int64_t n = d.n;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)c->sm_count * 8));
  k_action_angle<<<grid, 256, 0, c->stream>>>(d.vec, n, A, d_aa);
  CUDA_TRY(cudaGetLastError());
  c->launches++;
  CUDA_TRY(cudaMemcpyAsync(aa, d_aa, 6 * (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  return BMADGPU_OK;
}

// The cutoffs in effect: the list up to its first entry <= 0; all zero means the reference's
// default, one cutoff of 0.5 (lt_tracking_mod.f90:74).
int core_cutoffs(const bmadgpu_ltt_params* P, double* cut) {
  bool any = false;
  for (int i = 0; i < kCoreMax; i++) any = any || P->core_emit_cutoff[i] != 0;
  if (!any) {
    cut[0] = 0.5;
    return 1;
  }
  int n = 0;
  for (int i = 0; i < kCoreMax && P->core_emit_cutoff[i] > 0; i++) cut[n++] = P->core_emit_cutoff[i];
  return n;
}

int device_stats(bmadgpu_ctx* c, const bmadgpu_lattice* lat, const bmadgpu_bunch& d, double* d_scratch,
                 bmadgpu_bunch_data* bd) {
  double sums[kStatSums];
  CUDA_TRY(launch_bunch_sums(d.vec, d.t, d.state, d.n, d_scratch, d_scratch + kStatBlocks * kStatPass2, c->stream));
  c->launches += 4;
  CUDA_TRY(cudaMemcpyAsync(sums, d_scratch + kStatBlocks * kStatPass2, sizeof(sums), cudaMemcpyDeviceToHost,
                           c->stream));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  return bmadgpu_bunch_data_from_sums(sums, lat->param.p0c, lat->param.mass, bd);
}

}  // namespace

extern "C" int bmadgpu_bunch_stats(bmadgpu_ctx* c, const bmadgpu_lattice* lat, const bmadgpu_bunch* d,
                                   bmadgpu_bunch_data* bd) {
  if (!c || !lat || !d || !bd) return fail(BMADGPU_EINVAL, "NULL argument");
  if (d->n < 0 || (d->n > 0 && (!d->vec || !d->state))) return fail(BMADGPU_EINVAL, "bad bunch");
  CUDA_TRY(cudaSetDevice(c->device));
  double* scratch = nullptr;
  if (cudaMalloc(&scratch, sizeof(double) * (kStatBlocks * kStatPass2 + kStatSums)) != cudaSuccess)
    return fail(BMADGPU_ENOMEM, "cannot allocate statistics scratch");
  int r = device_stats(c, lat, *d, scratch, bd);
  cudaFree(scratch);
  return r;
}

extern "C" int bmadgpu_select_smallest(bmadgpu_ctx* c, const double* keys, int64_t n, int64_t n_cut,
                                       int32_t* mask, int32_t* selected) {
  if (!c || !keys || !mask || !selected) return fail(BMADGPU_EINVAL, "NULL argument");
  if (n < 1 || n_cut < 1 || n_cut > n) return fail(BMADGPU_EINVAL, "need 1 <= n_cut <= n");
  CUDA_TRY(cudaSetDevice(c->device));
  CoreScratch cs;
  if (!cs.alloc(n)) return fail(BMADGPU_ENOMEM, "cannot allocate the selection scratch");
  CUDA_TRY(cudaMemcpyAsync(cs.d_amp, keys, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  bool ok = false;
  int r = select_core(c, n, n_cut, cs, &ok);
  if (r) return r;
  if (ok)
    CUDA_TRY(cudaMemcpyAsync(mask, cs.d_mask, (size_t)n * sizeof(int32_t), cudaMemcpyDeviceToDevice, c->stream));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  *selected = ok ? 1 : 0;
  return BMADGPU_OK;
}

extern "C" int bmadgpu_bunch_core_emit(bmadgpu_ctx* c, const bmadgpu_lattice* lat, const bmadgpu_bunch* d,
                                       double cutoff, int32_t combined_calc, double* core_emit) {
  if (!c || !lat || !d || !core_emit) return fail(BMADGPU_EINVAL, "NULL argument");
  if (d->n < 1 || !d->vec || !d->state) return fail(BMADGPU_EINVAL, "bad bunch");
  if (!(cutoff > 0 && cutoff <= 1.00000001)) return fail(BMADGPU_EINVAL, "cutoff must be in (0, 1]");
  CUDA_TRY(cudaSetDevice(c->device));
  double* scratch = nullptr;
  if (cudaMalloc(&scratch, sizeof(double) * (kStatBlocks * kStatPass2 + kStatSums)) != cudaSuccess)
    return fail(BMADGPU_ENOMEM, "cannot allocate statistics scratch");
  bmadgpu_bunch_data bd;
  CoreScratch cs;
  int r = device_stats(c, lat, *d, scratch, &bd);
  if (!r) r = core_emittance(c, lat, *d, scratch, bd, cutoff, combined_calc != 0, cs, core_emit);
  cudaFree(scratch);
  return r;
}

extern "C" int bmadgpu_ltt_run(bmadgpu_ctx* c, const bmadgpu_lattice* lat, bmadgpu_bunch* hb,
                               const bmadgpu_ltt_params* P, int32_t* turns_done) {
  if (!c || !lat || !hb || !P) return fail(BMADGPU_EINVAL, "NULL argument");
  if (hb->n < 1 || !hb->vec || !hb->beta || !hb->state) return fail(BMADGPU_EINVAL, "bunch is empty or incomplete");
  if (P->n_turns < 0) return fail(BMADGPU_EINVAL, "n_turns < 0");
  if (lat->device != c->device) return fail(BMADGPU_EINVAL, "lattice and context are on different devices");
  CUDA_TRY(cudaSetDevice(c->device));
  const int64_t n = hb->n;
  const int n_ele = (int)lat->pk.info.n_ele;
  const std::string ave_base = P->averages_file ? P->averages_file : "";
  const std::string ps_base = P->phase_space_file ? P->phase_space_file : "";
  const std::string beam_base = P->beam_file ? P->beam_file : "";
  const std::string aa_base = P->action_angle_file ? P->action_angle_file : "";
  const std::string pp_base = P->per_particle_file ? P->per_particle_file : "";
  if (!pp_base.empty() && n > 1000)
    return fail(BMADGPU_EINVAL, "per-particle output needs at most 1000 particles (the reference stops there)");
  const bool particle_out = !ps_base.empty() || !aa_base.empty() || !pp_base.empty();
  if (P->ix_turn_start < 0 || P->ix_turn_start > P->n_turns) return fail(BMADGPU_EINVAL, "ix_turn_start out of range");
  // ltt_write_beam_file's schedule: every beam_every_n_turns turns, and always at n_turns
  auto wants_beam = [&](int turn) {
    if (beam_base.empty()) return false;
    const int nt = P->beam_every_n_turns;
    if (nt > 0 && P->output_only_last_turns > 0 && P->n_turns - turn >= P->output_only_last_turns) return false;
    if ((nt <= 0 || turn % nt != 0) && turn != P->n_turns) return false;
    return true;
  };
  const double cutoff = P->dead_cutoff > 0 ? P->dead_cutoff : 1.0;
  const int64_t dead_limit = (int64_t)std::llround(cutoff * (double)n);
  DevBunch cur, save;
  if (!cur.alloc(n) || !save.alloc(n)) return fail(BMADGPU_ENOMEM, "cannot allocate the device bunch");
  cudaStream_t s = c->stream;
  // loss records start as the host gives them (or unset)
  CUDA_TRY(cudaMemcpyAsync(cur.b.vec, hb->vec, 6 * n * sizeof(double), cudaMemcpyHostToDevice, s));
  CUDA_TRY(cudaMemcpyAsync(cur.b.beta, hb->beta, n * sizeof(double), cudaMemcpyHostToDevice, s));
  CUDA_TRY(cudaMemcpyAsync(cur.b.state, hb->state, n * sizeof(int32_t), cudaMemcpyHostToDevice, s));
  if (hb->t) CUDA_TRY(cudaMemcpyAsync(cur.b.t, hb->t, n * sizeof(double), cudaMemcpyHostToDevice, s));
  else CUDA_TRY(cudaMemsetAsync(cur.b.t, 0, n * sizeof(double), s));
  if (hb->ix_ele) CUDA_TRY(cudaMemcpyAsync(cur.b.ix_ele, hb->ix_ele, n * 4, cudaMemcpyHostToDevice, s));
  else CUDA_TRY(cudaMemsetAsync(cur.b.ix_ele, 0xff, n * 4, s));
  if (hb->ix_turn) CUDA_TRY(cudaMemcpyAsync(cur.b.ix_turn, hb->ix_turn, n * 4, cudaMemcpyHostToDevice, s));
  else CUDA_TRY(cudaMemsetAsync(cur.b.ix_turn, 0xff, n * 4, s));
  if (hb->location) CUDA_TRY(cudaMemcpyAsync(cur.b.location, hb->location, n * 4, cudaMemcpyHostToDevice, s));
  else CUDA_TRY(cudaMemsetAsync(cur.b.location, 0, n * 4, s));
  constexpr int kChunk = 1024;   // turns per moments buffer
  double *d_mom = nullptr, *d_scratch = nullptr;
  if (cudaMalloc(&d_mom, sizeof(double) * kChunk * BMADGPU_N_MOMENTS) != cudaSuccess ||
      cudaMalloc(&d_scratch, sizeof(double) * (kStatBlocks * kStatPass2 + kStatSums)) != cudaSuccess) {
    cudaFree(d_mom);
    return fail(BMADGPU_ENOMEM, "cannot allocate the moments buffer");
  }
  struct Freer {
    double* a;
    double* b;
    ~Freer() {
      cudaFree(a);
      cudaFree(b);
    }
  } freer{d_mom, d_scratch};
  std::vector<double> mom(kChunk * BMADGPU_N_MOMENTS);
  std::vector<double> hvec;
  std::vector<double> hbeta, ht;
  std::vector<int32_t> hstate;
  const std::string pre = preheader(lat, P);
  double cuts[kCoreMax];
  for (int i = 0; i < kCoreMax; i++)
    if (P->core_emit_cutoff[i] > 1.00000001) return fail(BMADGPU_EINVAL, "core_emit_cutoff must be <= 1");
  const int n_cuts = core_cutoffs(P, cuts);
  CoreScratch core_scratch;
  if (!ave_base.empty() && !write_averages_headers(ave_base, pre, cuts, n_cuts))
    return fail(BMADGPU_EINVAL, "cannot write the averages files " + ave_base + ".*");
  if (!pp_base.empty() && !write_per_particle_headers(pp_base, n, pre))
    return fail(BMADGPU_EINVAL, "cannot write the per-particle files " + pp_base);
  double* d_aa = nullptr;
  std::vector<double> haa;
  struct AaFreer {
    double** p;
    ~AaFreer() { cudaFree(*p); }
  } aa_freer{&d_aa};
  if (!aa_base.empty() && cudaMalloc(&d_aa, 6 * (size_t)n * sizeof(double)) != cudaSuccess)
    return fail(BMADGPU_ENOMEM, "cannot allocate the action-angle buffer");

  auto outputs = [&](int turn) -> int {
    if (!ave_base.empty() && wants(P->averages_every_n_turns, P->output_only_last_turns, P->n_turns, turn)) {
      bmadgpu_bunch_data bd;
      int r = device_stats(c, lat, cur.b, d_scratch, &bd);
      if (r) return r;
      double core[kCoreMax * 3];
      for (int k = 0; k < n_cuts; k++)
        if ((r = core_emittance(c, lat, cur.b, d_scratch, bd, cuts[k], P->core_emit_per_mode == 0, core_scratch,
                                core + 3 * k)))
          return r;
      if (!append_averages(ave_base, turn, bd, core, n_cuts))
        return fail(BMADGPU_EINVAL, "cannot append to the averages files");
    }
    if (!particle_out || !wants(P->particle_every_n_turns, P->output_only_last_turns, P->n_turns, turn))
      return BMADGPU_OK;
    if (!ps_base.empty() || !pp_base.empty()) {
      hvec.resize(6 * n);
      ht.resize(n);
      hstate.resize(n);
      bmadgpu_bunch h = *hb;
      h.vec = hvec.data();
      h.t = ht.data();
      h.state = hstate.data();
      CUDA_TRY(cudaMemcpyAsync(h.vec, cur.b.vec, 6 * n * sizeof(double), cudaMemcpyDeviceToHost, s));
      CUDA_TRY(cudaMemcpyAsync(h.t, cur.b.t, n * sizeof(double), cudaMemcpyDeviceToHost, s));
      CUDA_TRY(cudaMemcpyAsync(h.state, cur.b.state, n * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
      CUDA_TRY(cudaStreamSynchronize(s));
      if (!ps_base.empty() &&
          !write_phase_space(ps_base, turn, P->n_turns, h, lat->param.p0c, P->only_live_particles_out != 0, pre))
        return fail(BMADGPU_EINVAL, "cannot write the phase-space file");
      if (!pp_base.empty() && !append_per_particle(pp_base, turn, h, lat->param.p0c))
        return fail(BMADGPU_EINVAL, "cannot append to the per-particle files");
    }
    if (!aa_base.empty()) {
      bmadgpu_bunch_data bd;
      std::memset(&bd, 0, sizeof bd);
      int r = P->action_angle_n_inv ? BMADGPU_OK : device_stats(c, lat, cur.b, d_scratch, &bd);
      if (r) return r;
      haa.resize(6 * n);
      hstate.resize(n);
      if ((r = action_angle(c, cur.b, bd, P->action_angle_n_inv, d_aa, haa.data()))) return r;
      CUDA_TRY(cudaMemcpyAsync(hstate.data(), cur.b.state, n * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
      CUDA_TRY(cudaStreamSynchronize(s));
      if (!write_action_angle(aa_base, turn, P->n_turns, haa.data(), hstate.data(), n,
                              P->only_live_particles_out != 0, pre))
        return fail(BMADGPU_EINVAL, "cannot write the action-angle file");
    }
    return BMADGPU_OK;
  };
  auto beam_output = [&](int turn) -> int {
    if (!wants_beam(turn)) return BMADGPU_OK;
    std::vector<double> bv(6 * n), bb(n), bt(n);
    std::vector<int32_t> bs(n), be(n), bl(n);
    bmadgpu_bunch h;
    h.n = n;
    h.vec = bv.data();
    h.beta = bb.data();
    h.t = bt.data();
    h.state = bs.data();
    h.ix_ele = be.data();
    h.ix_turn = nullptr;
    h.location = bl.data();
    CUDA_TRY(cudaMemcpyAsync(h.vec, cur.b.vec, 6 * n * sizeof(double), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaMemcpyAsync(h.beta, cur.b.beta, n * sizeof(double), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaMemcpyAsync(h.t, cur.b.t, n * sizeof(double), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaMemcpyAsync(h.state, cur.b.state, n * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaMemcpyAsync(h.ix_ele, cur.b.ix_ele, n * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaMemcpyAsync(h.location, cur.b.location, n * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    // "<stem>-<turn, zero-padded to the digits of n_turns><.ext>"
    const int width = (int)std::log10(P->n_turns + 0.1) + 1;
    std::string num = std::to_string(turn);
    if ((int)num.size() < width) num = std::string(width - num.size(), '0') + num;
    std::string name;
    const size_t dot = beam_base.find_last_of('.');
    name = dot == std::string::npos ? beam_base + "-" + num : beam_base.substr(0, dot) + "-" + num + beam_base.substr(dot);
    if (bmadgpu_beam_write_file(name.c_str(), &h, &lat->param, 0.0, P->beam_exact ? BMADGPU_BEAM_EXACT : 0))
      return fail(BMADGPU_EINVAL, "cannot write the beam file " + name);
    return BMADGPU_OK;
  };

  int r = P->ix_turn_start == 0 ? outputs(0) : BMADGPU_OK;
  if (r) return r;
  int turn = P->ix_turn_start;
  bool stopped = false;
  while (turn < P->n_turns && !stopped) {
    int next = turn + 1;
    while (next < P->n_turns && next - turn < kChunk &&
           !(wants(P->averages_every_n_turns, P->output_only_last_turns, P->n_turns, next) && !ave_base.empty()) &&
           !(wants(P->particle_every_n_turns, P->output_only_last_turns, P->n_turns, next) && particle_out) &&
           !wants_beam(next))
      ++next;
    const int chunk = next - turn;
    CUDA_TRY(copy_bunch(save.b, cur.b, cudaMemcpyDeviceToDevice, s, true, true));
    if ((r = track_device(c, lat, &cur.b, 0, n_ele, turn, chunk, d_mom))) return r;
    CUDA_TRY(cudaMemcpyAsync(mom.data(), d_mom, sizeof(double) * chunk * BMADGPU_N_MOMENTS, cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    int stop_at = -1;
    for (int k = 0; k < chunk; k++) {
      const int64_t live = (int64_t)std::llround(mom[(size_t)k * BMADGPU_N_MOMENTS]);
      if (live == 0 || n - live >= dead_limit) {
        stop_at = k;
        break;
      }
    }
    if (stop_at >= 0) {
      stopped = true;
      if (stop_at < chunk - 1) {  // re-run exactly to the stopping turn
        CUDA_TRY(copy_bunch(cur.b, save.b, cudaMemcpyDeviceToDevice, s, true, true));
        if ((r = track_device(c, lat, &cur.b, 0, n_ele, turn, stop_at + 1, nullptr))) return r;
      }
      turn += stop_at + 1;
      break;
    }
    turn = next;
    if ((r = outputs(turn))) return r;
    if ((r = beam_output(turn))) return r;
  }
  // final state back to the caller
  bmadgpu_bunch out = *hb;
  CUDA_TRY(cudaMemcpyAsync(out.vec, cur.b.vec, 6 * n * sizeof(double), cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaMemcpyAsync(out.beta, cur.b.beta, n * sizeof(double), cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaMemcpyAsync(out.state, cur.b.state, n * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  if (out.t) CUDA_TRY(cudaMemcpyAsync(out.t, cur.b.t, n * sizeof(double), cudaMemcpyDeviceToHost, s));
  if (out.ix_ele) CUDA_TRY(cudaMemcpyAsync(out.ix_ele, cur.b.ix_ele, n * 4, cudaMemcpyDeviceToHost, s));
  if (out.ix_turn) CUDA_TRY(cudaMemcpyAsync(out.ix_turn, cur.b.ix_turn, n * 4, cudaMemcpyDeviceToHost, s));
  if (out.location) CUDA_TRY(cudaMemcpyAsync(out.location, cur.b.location, n * 4, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  if (turns_done) *turns_done = turn;
  return check_err_flag(c);
}
