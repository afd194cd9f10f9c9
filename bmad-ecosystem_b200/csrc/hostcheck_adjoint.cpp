// hostcheck_adjoint.cpp -- TEST-ONLY host build of the adjoint code (adjoint.cuh).
//
// Lets the CPU test suite check every element's vector-Jacobian product against finite
// differences of the same element's forward map, and the whole per-particle adjoint sweep
// (checkpoints, turn and element recomputation) against finite differences of the oracle,
// without a GPU. Built into _build/libbmadgpu_hostadjoint.so, which the product never loads.

#include <cstring>
#include <string>
#include <vector>

#include "../../include/bmadgpu.h"
#include "adjoint.cuh"
#include "lattice.h"

using namespace bmadgpu;

namespace bmadgpu {
double h_cmulti[kNPole][kNPole];
double h_cfull[kNPole][kNPole];
}  // namespace bmadgpu

namespace {
thread_local std::string g_err;

Globals host_globals(const bmadgpu_param& p) {
  Globals g;
  g.p0c = p.p0c;
  g.e_tot = p.e_tot;
  g.mass = p.mass;
  g.beta0 = p.p0c / p.e_tot;
  g.max_ap = p.max_aperture_limit;
  g.mass2 = p.mass * p.mass;
  double me = p.mass / p.e_tot;
  g.lez_me2 = me * me;
  g.lez_b02 = g.beta0 * g.beta0;
  g.lez_f = g.lez_b02 * (2 * g.lez_b02 - g.lez_me2 / 2);
  g.lez_thresh = 3e-7 * p.e_tot;
  g.charge = p.charge;
  g.inv_beta0 = 1 / g.beta0;
  return g;
}

struct Packed {
  PackedLattice pk;
  const EleHdr* hdr;
  const ApRec* ap;
  const double* pool;
  Globals G;
};

int pack(const bmadgpu_element* eles, int32_t n, const bmadgpu_param* param, Packed& P) {
  static bool tables = false;
  if (!tables) {
    build_cmulti_tables(h_cmulti, h_cfull);
    tables = true;
  }
  int r = pack_lattice(eles, n, *param, P.pk, g_err);
  if (r) return r;
  const uint8_t* tbl = P.pk.image.data();
  P.hdr = reinterpret_cast<const EleHdr*>(tbl);
  P.ap = reinterpret_cast<const ApRec*>(tbl + P.pk.info.hdr_bytes);
  P.pool = reinterpret_cast<const double*>(tbl + P.pk.info.hdr_bytes + P.pk.info.ap_bytes);
  P.G = host_globals(*param);
  return 0;
}

void to_particle(const double* s, Particle& p, const Globals& G) {
  p.x = s[0];
  p.px = s[1];
  p.y = s[2];
  p.py = s[3];
  p.z = s[4];
  p.pz = s[5];
  p.beta = s[6];
  p.state = S_ALIVE;
  refresh(p, G);
}
}  // namespace

extern "C" {

const char* bmadgpu_hostadjoint_last_error(void) { return g_err.c_str(); }

// Element ie of the lattice on state s[7] (x, px, y, py, z, pz, beta): out[7]; returns the
// particle state code.
int bmadgpu_hostadjoint_element_track(const bmadgpu_element* eles, int32_t n, const bmadgpu_param* param, int32_t ie,
                                      const double* s, double* out) {
  Packed P;
  int r = pack(eles, n, param, P);
  if (r) return r;
  Particle p;
  to_particle(s, p, P.G);
  track1(p, P.hdr[ie], P.pool, P.ap, P.G, false);
  out[0] = p.x; out[1] = p.px; out[2] = p.y; out[3] = p.py; out[4] = p.z; out[5] = p.pz; out[6] = p.beta;
  return p.state;
}

// Vector-Jacobian product of element ie at s[7]: lam[7] (output cotangent) -> input cotangent,
// *gscale = sum over strength coefficients c of c dL/dc. Returns 1 if the element is outside
// the adjoint path.
int bmadgpu_hostadjoint_element_vjp(const bmadgpu_element* eles, int32_t n, const bmadgpu_param* param, int32_t ie,
                                    const double* s, double* lam, double* gscale) {
  Packed P;
  int r = pack(eles, n, param, P);
  if (r) return r;
  if (adj_supported(P.hdr[ie])) return 1;
  Particle p;
  to_particle(s, p, P.G);
  Adj a = {lam[0], lam[1], lam[2], lam[3], lam[4], lam[5], lam[6]};
  double gs = 0;
  vjp_element(P.hdr[ie], P.pool, p, a, gs, P.G);
  lam[0] = a.x; lam[1] = a.px; lam[2] = a.y; lam[3] = a.py; lam[4] = a.z; lam[5] = a.pz; lam[6] = a.beta;
  *gscale = gs;
  return 0;
}

// The whole adjoint on the CPU with the device driver (adj_particle): loss and, per slot, the
// scale derivative sum_c c dL/dc summed over particles. param_of_ele[n_ele] gives each element's
// slot (-1: none). The bunch is updated to its state after n_turns.
int bmadgpu_hostadjoint_loss_grad(const bmadgpu_element* eles, int32_t n_ele, const bmadgpu_param* param,
                                  bmadgpu_bunch* b, int32_t n_turns, int32_t every, int32_t n_slot,
                                  const int32_t* param_of_ele, double* loss, double* gscale) {
  Packed P;
  int r = pack(eles, n_ele, param, P);
  if (r) return r;
  for (int32_t i = 0; i < n_ele; i++)
    if (param_of_ele[i] >= 0 && adj_supported(P.hdr[i])) return BMADGPU_EUNSUPPORTED;
  const int64_t N = b->n;
  const int n_seg = (n_turns + every - 1) / every;
  std::vector<double> ckpt((size_t)n_seg * 7 * N), turnbuf((size_t)every * 7 * N), elebuf((size_t)n_ele * 7 * N),
      gradbuf((size_t)n_slot * N, 0.0), lossbuf(N);
  AdjArgs a;
  a.hdr = P.hdr;
  a.ap = P.ap;
  a.pool = P.pool;
  a.n_ele = n_ele;
  a.n_turns = n_turns;
  a.every = every;
  a.N = N;
  a.G = P.G;
  a.param_of_ele = param_of_ele;
  a.ckpt = ckpt.data();
  a.turnbuf = turnbuf.data();
  a.elebuf = elebuf.data();
  a.gradbuf = gradbuf.data();
  a.lossbuf = lossbuf.data();
  a.vec = b->vec;
  a.beta = b->beta;
  a.state = b->state;
  a.loss_scale = 1.0 / (double)N;
  for (int64_t j = 0; j < N; j++) adj_particle(a, j);
  double L = 0;
  for (int64_t j = 0; j < N; j++) L += lossbuf[j];
  *loss = L;
  for (int32_t s = 0; s < n_slot; s++) {
    double g = 0;
    for (int64_t j = 0; j < N; j++) g += gradbuf[(size_t)s * N + j];
    gscale[s] = g;
  }
  return 0;
}

}  // extern "C"
