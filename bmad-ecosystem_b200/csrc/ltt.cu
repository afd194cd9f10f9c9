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

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
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

bool write_averages_headers(const std::string& base, const std::string& pre) {
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
  std::fprintf(f, "%s%s\n%s\n", pre.c_str(), l1.c_str(), l2.c_str());
  std::fclose(f);
  return true;
}

bool append_averages(const std::string& base, int turn, const bmadgpu_bunch_data& bd) {
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
  std::fprintf(f, "%s\n", l.c_str());
  std::fclose(f);
  return true;
}

bool write_phase_space(const std::string& base, int turn, int n_turns, const bmadgpu_bunch& h, double p0c,
                       bool only_live, const std::string& pre) {
  std::string num;
  if (n_turns > 0) {
    const int width = (int)(std::log10((double)n_turns) + 1 + 1e-10);
    char b[32];
    std::snprintf(b, sizeof b, "%0*d", width, turn);
    num = b;
  } else {
    num = "000";
  }
  std::string name;
  size_t ix = base.find('#');
  name = ix == std::string::npos ? base + num : base.substr(0, ix) + num + base.substr(ix + 1);
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
  if (!ave_base.empty() && !write_averages_headers(ave_base, pre))
    return fail(BMADGPU_EINVAL, "cannot write the averages files " + ave_base + ".*");

  auto outputs = [&](int turn) -> int {
    if (!ave_base.empty() && wants(P->averages_every_n_turns, P->output_only_last_turns, P->n_turns, turn)) {
      bmadgpu_bunch_data bd;
      int r = device_stats(c, lat, cur.b, d_scratch, &bd);
      if (r) return r;
      if (!append_averages(ave_base, turn, bd)) return fail(BMADGPU_EINVAL, "cannot append to the averages files");
    }
    if (!ps_base.empty() && wants(P->particle_every_n_turns, P->output_only_last_turns, P->n_turns, turn)) {
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
      if (!write_phase_space(ps_base, turn, P->n_turns, h, lat->param.p0c, P->only_live_particles_out != 0, pre))
        return fail(BMADGPU_EINVAL, "cannot write the phase-space file");
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
    if (bmadgpu_beam_write_ascii(name.c_str(), &h, &lat->param, 0.0, P->beam_exact ? BMADGPU_BEAM_EXACT : 0))
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
           !(wants(P->particle_every_n_turns, P->output_only_last_turns, P->n_turns, next) && !ps_base.empty()) &&
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
