// bunchdata.cpp -- bunch data of the long-term-tracking outputs from the device sums (host side).
//
// Restates, on the sums of stats.cu:
//   ltt_calc_bunch_data            bsim/modules/lt_tracking_mod.f90:2369-2421 (sigma_vec with the
//                                  round-off zeroing rule, sig1, skewness, kurtosis)
//   calc_bunch_params              bmad/multiparticle/beam_utils.f90:1326-1431 (centroid, t, sigma_t)
//   calc_emittances_and_twiss_from_sigma_matrix  beam_utils.f90:1454-1690 (projected x/y/z Twiss
//                                  and emittances; normal-mode emittances a, b, c = the eigenvalues
//                                  +-i emit of sigma.S, modes sorted as mat_eigen sorts them,
//                                  sim_utils/matrix/mat_eigen.f90:37-187)
// The eigenvalues of sigma.S are found as those of L^T S L (sigma = L L^T), a real antisymmetric
// matrix, through the real symmetric form [[0, -A], [A, 0]] and a cyclic Jacobi iteration; the
// eigenvectors of sigma.S are L w. The reference uses LAPACK's geev on sigma.S directly.

#include <cmath>
#include <complex>
#include <cstring>

#include "../../include/bmadgpu.h"
#include "stats.cuh"

namespace {

// Cyclic Jacobi on a real symmetric n x n matrix (row-major): eigenvalues in d, eigenvectors as
// the columns of v.
void jacobi_sym(int n, double* a, double* d, double* v) {
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) v[i * n + j] = (i == j) ? 1.0 : 0.0;
  for (int sweep = 0; sweep < 100; sweep++) {
    double off = 0, diag = 0;
    for (int i = 0; i < n; i++)
      for (int j = 0; j < n; j++) (i == j ? diag : off) += a[i * n + j] * a[i * n + j];
    if (off <= 1e-30 * diag || off == 0) break;
    for (int p = 0; p < n - 1; p++)
      for (int q = p + 1; q < n; q++) {
        const double apq = a[p * n + q];
        if (apq == 0) continue;
        const double app = a[p * n + p], aqq = a[q * n + q];
        const double theta = (aqq - app) / (2 * apq);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1));
        const double c = 1 / std::sqrt(t * t + 1), s = t * c;
        for (int k = 0; k < n; k++) {
          const double akp = a[k * n + p], akq = a[k * n + q];
          a[k * n + p] = c * akp - s * akq;
          a[k * n + q] = s * akp + c * akq;
        }
        for (int k = 0; k < n; k++) {
          const double apk = a[p * n + k], aqk = a[q * n + k];
          a[p * n + k] = c * apk - s * aqk;
          a[q * n + k] = s * apk + c * aqk;
        }
        for (int k = 0; k < n; k++) {
          const double vkp = v[k * n + p], vkq = v[k * n + q];
          v[k * n + p] = c * vkp - s * vkq;
          v[k * n + q] = s * vkp + c * vkq;
        }
      }
  }
  for (int i = 0; i < n; i++) d[i] = a[i * n + i];
}

// N of calc_emittances_and_twiss_from_sigma_matrix (bmad/multiparticle/beam_utils.f90:1495-1551)
// from the Jacobi eigenvectors. For the Jacobi pair (x, y) of eigenvalue d, w = x + i y satisfies
// A w = -i d w, so v = L w is the eigenvector of sigma.S at -i d: the vector geev's pair gives
// mat_eigen before its flip (mat_eigen.f90:149-150). Then, as there and in normalize_e (:1639-1688):
// the flip to positive fnorm = sum 2 Im(conj(v_2k) v_2k+1) (:153-164), the phase that makes the
// mode's own-plane component real and positive (:175-182), e_odd = conj(e_even) with e_even
// scaled by sqrt(i)/sqrt(wronskian), and N = E Q with Wolski's Q, whose real entries are the
// single-precision 1.0/sqrt(2.0) and whose imaginary ones are i / (single-precision sqrt(2.0)).
void normal_form_matrix(const double* L, const double* V, int n2, int dim, int nm, const int* col,
                        const int* sort, double* nmat) {
  typedef std::complex<double> cd;
  const double q_re = (double)(1.0f / std::sqrt(2.0f));
  const double q_im = 1.0 / (double)std::sqrt(2.0f);
  for (int i = 0; i < 36; i++) nmat[i] = 0;
  if (dim == 4) nmat[28] = nmat[35] = 1;
  for (int m = 0; m < nm; m++) {
    const int b = col[m], p = sort[m];
    cd v[6];
    for (int c = 0; c < dim; c++) {
      double vr = 0, vi = 0;
      for (int k = 0; k < dim; k++) {
        vr += L[c * 6 + k] * V[k * n2 + b];
        vi += L[c * 6 + k] * V[(dim + k) * n2 + b];
      }
      v[c] = cd(vr, vi);
    }
    double fnorm = 0;
    for (int c = 0; c < dim; c += 2) fnorm += 2 * (std::conj(v[c]) * v[c + 1]).imag();
    if (fnorm < 0) {
      for (int c = 0; c < dim; c++) v[c] = std::conj(v[c]);
      fnorm = -fnorm;
    }
    const cd vk = v[2 * p];
    const cd sgn = std::abs(vk) == 0 ? cd(1 / std::sqrt(fnorm), 0) : std::abs(vk) / (std::sqrt(fnorm) * vk);
    cd e1[6], e2[6];
    for (int c = 0; c < dim; c++) {
      e1[c] = sgn * v[c];
      e2[c] = std::conj(e1[c]);
    }
    // normalize_e: wronskian of (conj(e2), S e2), S = blocks [[0, 1], [-1, 0]]
    cd wr = 0;
    for (int c = 0; c < dim; c += 2) wr += std::conj(e2[c]) * e2[c + 1] - std::conj(e2[c + 1]) * e2[c];
    const cd factor = std::sqrt(cd(0, 1)) / std::sqrt(wr);
    for (int c = 0; c < dim; c++) {
      e2[c] *= factor;
      e1[c] = std::conj(e2[c]);
    }
    for (int c = 0; c < dim; c++) {
      nmat[c * 6 + 2 * p] = (e1[c] * q_re + e2[c] * q_re).real();
      nmat[c * 6 + 2 * p + 1] = (e1[c] * cd(0, q_im) + e2[c] * cd(0, -q_im)).real();
    }
  }
}

// Normal-mode emittances of the centred sigma matrix (dim 4 or 6) and, if nmat is not NULL, the
// normal-form matrix N of calc_emittances_and_twiss_from_sigma_matrix (6x6 row-major, Wolski
// Eq. 44; in dim 4 its longitudinal block is the identity, where the reference leaves it unset).
// Returns false if sigma is not positive definite (the reference's eigen-analysis then fails as
// well).
bool normal_mode_emittances(const double* sig, int dim, double* emit, double* nmat) {
  double L[36] = {0};
  for (int j = 0; j < dim; j++) {
    double s = sig[j * 6 + j];
    for (int k = 0; k < j; k++) s -= L[j * 6 + k] * L[j * 6 + k];
    if (!(s > 0)) return false;
    L[j * 6 + j] = std::sqrt(s);
    for (int i = j + 1; i < dim; i++) {
      double t = sig[i * 6 + j];
      for (int k = 0; k < j; k++) t -= L[i * 6 + k] * L[j * 6 + k];
      L[i * 6 + j] = t / L[j * 6 + j];
    }
  }
  // A = L^T S L, S = blocks [[0, 1], [-1, 0]]
  double SL[36] = {0}, A[36] = {0};
  for (int i = 0; i < dim; i += 2)
    for (int k = 0; k < dim; k++) {
      SL[i * 6 + k] = L[(i + 1) * 6 + k];
      SL[(i + 1) * 6 + k] = -L[i * 6 + k];
    }
  for (int i = 0; i < dim; i++)
    for (int j = 0; j < dim; j++) {
      double s = 0;
      for (int k = 0; k < dim; k++) s += L[k * 6 + i] * SL[k * 6 + j];
      A[i * 6 + j] = s;
    }
  const int n2 = 2 * dim;
  double B[144] = {0}, d[12], V[144];
  for (int i = 0; i < dim; i++)
    for (int j = 0; j < dim; j++) {
      B[i * n2 + (dim + j)] = -A[i * 6 + j];
      B[(dim + i) * n2 + j] = A[i * 6 + j];
    }
  jacobi_sym(n2, B, d, V);
  // the dim/2 largest eigenvalues (each appears twice) are the emittances; one eigenvector each
  const int nm = dim / 2;
  int used[12] = {0}, used_first[3] = {0};
  double eps[3] = {0}, amp[3][3] = {{0}};
  for (int m = 0; m < nm; m++) {
    int best = -1;
    for (int i = 0; i < n2; i++)
      if (!used[i] && (best < 0 || d[i] > d[best])) best = i;
    used[best] = 1;
    used_first[m] = best;
    // mark its twin (the other eigenvector of the same value) as used
    int twin = -1;
    for (int i = 0; i < n2; i++)
      if (!used[i] && (twin < 0 || std::fabs(d[i] - d[best]) < std::fabs(d[twin] - d[best]))) twin = i;
    if (twin >= 0) used[twin] = 1;
    eps[m] = d[best];
    // eigenvector of sigma.S: v = L (x + i y), |v_c|^2 per plane
    double x[6], y[6];
    for (int k = 0; k < dim; k++) {
      x[k] = V[k * n2 + best];
      y[k] = V[(dim + k) * n2 + best];
    }
    double tot = 0;
    for (int pl = 0; pl < nm; pl++) {
      double s = 0;
      for (int c = 2 * pl; c < 2 * pl + 2; c++) {
        double vr = 0, vi = 0;
        for (int k = 0; k < dim; k++) {
          vr += L[c * 6 + k] * x[k];
          vi += L[c * 6 + k] * y[k];
        }
        s += vr * vr + vi * vi;
      }
      amp[pl][m] = s;
      tot += s;
    }
    for (int pl = 0; pl < nm; pl++) amp[pl][m] /= tot;
  }
  // mat_eigen's greedy assignment of modes to planes
  int sort[3] = {0, 1, 2};
  for (int it = 0; it < nm; it++) {
    double dmax[3];
    for (int j = 0; j < nm; j++) {
      int m1 = 0;
      for (int i = 1; i < nm; i++)
        if (amp[j][i] > amp[j][m1]) m1 = i;
      double second = -1;
      for (int i = 0; i < nm; i++)
        if (i != m1 && amp[j][i] > second) second = amp[j][i];
      if (nm == 1) second = -1;
      dmax[j] = amp[j][m1] - second;
    }
    int k = 0;
    for (int j = 1; j < nm; j++)
      if (dmax[j] > dmax[k]) k = j;
    int m = 0;
    for (int i = 1; i < nm; i++)
      if (amp[k][i] > amp[k][m]) m = i;
    sort[m] = k;
    for (int i = 0; i < nm; i++) amp[k][i] = 0;
    for (int j = 0; j < nm; j++) amp[j][m] = 0;
  }
  for (int m = 0; m < 3; m++) emit[m] = 0;
  for (int m = 0; m < nm; m++) emit[sort[m]] = eps[m];
  if (nmat) normal_form_matrix(L, V, n2, dim, nm, used_first, sort, nmat);
  return true;
}

}  // namespace

extern "C" int bmadgpu_bunch_data_from_sums(const double* s, double p0c, double mass, bmadgpu_bunch_data* bd) {
  if (!s || !bd) return BMADGPU_EINVAL;
  std::memset(bd, 0, sizeof(*bd));
  const double n = s[0];
  bd->n_live = (int64_t)n;
  bd->p0c = p0c;
  if (n <= 0) return BMADGPU_OK;
  const double* sv = s + 1;      // sum v_i
  const double* s2 = s + 9;      // sum v_i v_j, i <= j
  const double* c2 = s + bmadgpu::kStatPass1;        // centred sums
  const double* c3 = c2 + 21;
  const double* c4 = c2 + 27;
  // calc_bunch_params: centroid, t, sigma_t, centred sigma matrix
  for (int i = 0; i < 6; i++) bd->centroid[i] = sv[i] / n;
  bd->t = s[7] / n;
  bd->sigma_t = std::sqrt(std::fmax(0.0, s[8] / n - bd->t * bd->t));
  int k = 0;
  for (int i = 0; i < 6; i++)
    for (int j = i; j < 6; j++, k++) {
      bd->sigma[i * 6 + j] = bd->sigma[j * 6 + i] = c2[k] / n;
    }
  // projected Twiss (projected_twiss_calc)
  const double* S = bd->sigma;
  const double s66 = S[35];
  const double f_emit = p0c * (1.0 + bd->centroid[5]) / mass;
  const int pl[3][5] = {{0, 7, 1, 5, 11}, {14, 21, 15, 17, 23}, {28, 35, 29, -1, -1}};
  for (int p = 0; p < 3; p++) {
    const double x2_0 = S[pl[p][0]], px2_0 = S[pl[p][1]], xpx_0 = S[pl[p][2]];
    const double xd = pl[p][3] >= 0 ? S[pl[p][3]] : 0.0, pxd = pl[p][4] >= 0 ? S[pl[p][4]] : 0.0;
    double x2 = x2_0, xpx = xpx_0, px2 = px2_0;
    if (s66 != 0) {
      if (p < 2) {
        bd->eta[p] = xd / s66;
        bd->etap[p] = pxd / s66;
      }
      x2 = x2_0 - xd * xd / s66;
      xpx = xpx_0 - xd * pxd / s66;
      px2 = px2_0 - pxd * pxd / s66;
    }
    const double e = std::sqrt(std::fmax(0.0, x2 * px2 - xpx * xpx));
    bd->proj_emit[p] = e;
    if (e != 0) {
      bd->proj_alpha[p] = -xpx / e;
      bd->proj_beta[p] = x2 / e;
    }
  }
  // normal modes (n_live >= 6)
  if (n >= 6) {
    double mx = 0;
    for (int i = 0; i < 36; i++) mx = std::fmax(mx, std::fabs(S[i]));
    const double cut = 1e-20 * mx;
    const int dim = (std::fabs(S[28]) < cut || std::fabs(S[35]) < cut) ? 4 : 6;
    bd->emit_valid = normal_mode_emittances(S, dim, bd->emit, nullptr) ? 1 : 0;
    for (int m = 0; m < 3; m++) bd->norm_emit[m] = bd->emit[m] * f_emit;
  }
  // ltt_calc_bunch_data (needs at least 10 live particles)
  if (n < 10) return BMADGPU_OK;
  k = 0;
  for (int i = 0; i < 6; i++)
    for (int j = i; j < 6; j++, k++) {
      double v = s2[k] / n - sv[i] * sv[j] / (n * n);
      if (std::fabs(v) < 1e-15 * std::fabs(sv[i] * sv[j]) / n) v = 0;
      bd->sigma_vec[k] = v;
      if (i == j) bd->sig1[i] = std::sqrt(std::fmax(0.0, v));
    }
  for (int p = 0; p < 3; p++) {
    const int i = 2 * p;
    const double sg = bd->sig1[i];
    if (sg != 0) {
      bd->skew[p] = c3[i] / (n * (sg * sg * sg));
      bd->kurt[p] = c4[i] / (n * (sg * sg * sg * sg)) - 3.0;
    }
  }
  return BMADGPU_OK;
}

extern "C" int bmadgpu_sigma_normal_form(const double* sigma, double* emit, double* n_mat) {
  if (!sigma || !n_mat) return BMADGPU_EINVAL;
  double mx = 0;
  for (int i = 0; i < 36; i++) mx = std::fmax(mx, std::fabs(sigma[i]));
  const double cut = 1e-20 * mx;
  const int dim = (std::fabs(sigma[28]) < cut || std::fabs(sigma[35]) < cut) ? 4 : 6;
  double e[3];
  if (!normal_mode_emittances(sigma, dim, e, n_mat)) return BMADGPU_EINVAL;
  if (emit)
    for (int m = 0; m < 3; m++) emit[m] = e[m];
  return BMADGPU_OK;
}
