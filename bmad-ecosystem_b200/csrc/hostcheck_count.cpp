// hostcheck_count.cpp -- TEST/MEASUREMENT-ONLY: the device element code compiled for the host with
// every floating-point value replaced by a counting type, to obtain the algorithmic FP64
// operation count per particle-turn (the roofline numerator) from the very source the GPU runs.
// Counts: add/sub, mul, div, sqrt, and transcendental calls (sin, cos, asin, atan2, sinh, cosh, exp, tan,
// fmod, fma), each counted once.
#include <math.h>
#include <stdint.h>

#include <cmath>
#include <cstring>
#include <string>

#include "../../include/bmadgpu.h"
#include "lattice.h"
#include "table.h"

namespace bmadgpu {
struct OpCounts {
  double add, mul, div, sqrt, trans;
};
static thread_local OpCounts g_ops = {0, 0, 0, 0, 0};

struct CD {  // counted double
  double v;
  CD() : v(0) {}
  CD(double x) : v(x) {}
  CD(int x) : v(x) {}
  CD(unsigned x) : v(x) {}
  explicit operator double() const { return v; }
  explicit operator int() const { return (int)v; }
  CD& operator+=(CD o) { g_ops.add++; v += o.v; return *this; }
  CD& operator-=(CD o) { g_ops.add++; v -= o.v; return *this; }
  CD& operator*=(CD o) { g_ops.mul++; v *= o.v; return *this; }
  CD& operator/=(CD o) { g_ops.div++; v /= o.v; return *this; }
};
inline CD operator+(CD a, CD b) { g_ops.add++; return CD(a.v + b.v); }
inline CD operator-(CD a, CD b) { g_ops.add++; return CD(a.v - b.v); }
inline CD operator*(CD a, CD b) { g_ops.mul++; return CD(a.v * b.v); }
inline CD operator/(CD a, CD b) { g_ops.div++; return CD(a.v / b.v); }
inline CD operator-(CD a) { return CD(-a.v); }
#define BG_CMP(op) \
  inline bool operator op(CD a, CD b) { return a.v op b.v; } \
  inline bool operator op(CD a, double b) { return a.v op b; } \
  inline bool operator op(double a, CD b) { return a op b.v; } \
  inline bool operator op(CD a, int b) { return a.v op b; } \
  inline bool operator op(int a, CD b) { return a op b.v; }
BG_CMP(<) BG_CMP(>) BG_CMP(<=) BG_CMP(>=) BG_CMP(==) BG_CMP(!=)
#undef BG_CMP
#define BG_ARI(op) \
  inline CD operator op(CD a, double b) { return a op CD(b); } \
  inline CD operator op(double a, CD b) { return CD(a) op b; } \
  inline CD operator op(CD a, int b) { return a op CD(b); } \
  inline CD operator op(int a, CD b) { return CD(a) op b; }
BG_ARI(+) BG_ARI(-) BG_ARI(*) BG_ARI(/)
#undef BG_ARI
inline CD sqrt(CD a) { g_ops.sqrt++; return CD(std::sqrt(a.v)); }
inline CD fabs(CD a) { return CD(std::fabs(a.v)); }
inline CD sin(CD a) { g_ops.trans++; return CD(std::sin(a.v)); }
inline CD cos(CD a) { g_ops.trans++; return CD(std::cos(a.v)); }
inline CD asin(CD a) { g_ops.trans++; return CD(std::asin(a.v)); }
inline CD atan2(CD a, CD b) { g_ops.trans++; return CD(std::atan2(a.v, b.v)); }
inline CD sinh(CD a) { g_ops.trans++; return CD(std::sinh(a.v)); }
inline CD cosh(CD a) { g_ops.trans++; return CD(std::cosh(a.v)); }
inline CD exp(CD a) { g_ops.trans++; return CD(std::exp(a.v)); }
inline CD tan(CD a) { g_ops.trans++; return CD(std::tan(a.v)); }
inline CD fmod(CD a, CD b) { g_ops.trans++; return CD(std::fmod(a.v, b.v)); }
inline CD floor(CD a) { g_ops.trans++; return CD(std::floor(a.v)); }
inline CD fma(CD a, CD b, CD c) { g_ops.trans++; return CD(std::fma(a.v, b.v, c.v)); }
double h_cmulti_raw[22][22];
double h_cfull_raw[22][22];
}  // namespace bmadgpu

// The element code with every `double` counted. table.h (ApRec, Globals, EleHdr) is already
// included with plain doubles; the maps and particle state become counted.
#define double bmadgpu::CD
#define BG_COUNT_OPS
#define h_cmulti h_cmulti_c
#define h_cfull h_cfull_c
#include "elements.cuh"
#undef h_cmulti
#undef h_cfull
#undef double

namespace bmadgpu {
CD h_cmulti_c[kNPole][kNPole];
CD h_cfull_c[kNPole][kNPole];
}

using namespace bmadgpu;

extern "C" {

// Tracks n particles (host SoA) n_turns and returns the op counts summed over all particle-turns
// tracked: counts[0..4] = add/sub, mul, div, sqrt, transcendental; counts[5] = particle-turns.
int bmadgpu_hostcheck_count_ops(const bmadgpu_element* eles, int32_t n_ele, const bmadgpu_param* param,
                                bmadgpu_bunch* b, int32_t n_turns, double* counts) {
  static bool tables = false;
  if (!tables) {
    build_cmulti_tables(h_cmulti_raw, h_cfull_raw);
    for (int i = 0; i < kNPole; i++)
      for (int j = 0; j < kNPole; j++) {
        h_cmulti_c[i][j] = CD(h_cmulti_raw[i][j]);
        h_cfull_c[i][j] = CD(h_cfull_raw[i][j]);
      }
    tables = true;
  }
  PackedLattice pk;
  std::string err;
  int r = pack_lattice(eles, n_ele, *param, pk, err);
  if (r) return r;
  const uint8_t* tbl = pk.image.data();
  const EleHdr* hdr = reinterpret_cast<const EleHdr*>(tbl);
  const ApRec* ap = reinterpret_cast<const ApRec*>(tbl + pk.info.hdr_bytes);
  const CD* pool = reinterpret_cast<const CD*>(tbl + pk.info.hdr_bytes + pk.info.ap_bytes);
  Globals G;
  G.p0c = param->p0c; G.e_tot = param->e_tot; G.mass = param->mass; G.beta0 = param->p0c / param->e_tot;
  G.max_ap = param->max_aperture_limit; G.mass2 = param->mass * param->mass;
  double me = param->mass / param->e_tot;
  G.lez_me2 = me * me; G.lez_b02 = G.beta0 * G.beta0; G.lez_f = G.lez_b02 * (2 * G.lez_b02 - G.lez_me2 / 2);
  G.lez_thresh = 3e-7 * param->e_tot; G.charge = param->charge;
  G.inv_beta0 = 1 / G.beta0;
  g_ops = OpCounts{0, 0, 0, 0, 0};
  double pturns = 0;
  const int64_t n = b->n;
  for (int64_t j = 0; j < n; j++) {
    Particle p;
    p.x = b->vec[j]; p.px = b->vec[n + j]; p.y = b->vec[2 * n + j];
    p.py = b->vec[3 * n + j]; p.z = b->vec[4 * n + j]; p.pz = b->vec[5 * n + j];
    p.beta = b->beta[j];
    p.state = b->state[j];
    if (p.state != S_ALIVE) continue;
    refresh(p, G);
    bool lost = false;
    for (int turn = 0; turn < n_turns && !lost; turn++) {
      pturns += 1;
      for (int ie = 0; ie < n_ele; ie++) {
        if (track1(p, hdr[ie], pool, ap, G, turn == 0 && ie == 0)) { lost = true; break; }
      }
    }
  }
  counts[0] = g_ops.add; counts[1] = g_ops.mul; counts[2] = g_ops.div;
  counts[3] = g_ops.sqrt; counts[4] = g_ops.trans; counts[5] = pturns;
  return 0;
}

}  // extern "C"
