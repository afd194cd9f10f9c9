// capi.cu -- extern "C" entry points of include/bmadgpu.h.
//
// Contexts own a CUDA stream, device staging buffers for the host-pointer API, the
// live-particle lists used for loss compaction, and the launch tuning. Lattices own the packed
// element table in device memory. Nothing here keeps global mutable state except the
// thread-local last-error message.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>

#include "capi_internal.h"

using namespace bmadgpu;

namespace bmadgpu {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

int cuda_fail(cudaError_t e, const char* what) {
  return fail(BMADGPU_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

}  // namespace bmadgpu

namespace {

__global__ void k_set_i64(int64_t* p, int64_t v) { *p = v; }

int ensure_live(bmadgpu_ctx* c, int64_t n) {
  if (n <= c->live_cap) return BMADGPU_OK;
  for (int i = 0; i < 2; i++) {
    if (c->d_live[i]) cudaFree(c->d_live[i]);
    c->d_live[i] = nullptr;
  }
  c->live_cap = 0;
  for (int i = 0; i < 2; i++)
    if (cudaMalloc(&c->d_live[i], (size_t)n * sizeof(int32_t)) != cudaSuccess)
      return fail(BMADGPU_ENOMEM, "cannot allocate live-particle lists");
  c->live_cap = n;
  return BMADGPU_OK;
}

int ensure_staging(bmadgpu_ctx* c, int64_t n) {
  if (n <= c->cap) return BMADGPU_OK;
  cudaFree(c->d_vec);
  cudaFree(c->d_beta);
  cudaFree(c->d_t);
  cudaFree(c->d_i32);
  c->d_vec = nullptr; c->d_beta = nullptr; c->d_t = nullptr; c->d_i32 = nullptr;
  c->cap = 0;
  if (cudaMalloc(&c->d_vec, (size_t)n * 6 * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&c->d_beta, (size_t)n * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&c->d_t, (size_t)n * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&c->d_i32, (size_t)n * 4 * sizeof(int32_t)) != cudaSuccess)
    return fail(BMADGPU_ENOMEM, "cannot allocate device particle buffers");
  c->cap = n;
  return BMADGPU_OK;
}

int check_bunch(const bmadgpu_bunch* b) {
  if (!b) return fail(BMADGPU_EINVAL, "bunch is NULL");
  if (b->n < 0) return fail(BMADGPU_EINVAL, "bunch n < 0");
  if (b->n > 0 && (!b->vec || !b->beta || !b->state)) return fail(BMADGPU_EINVAL, "bunch vec/beta/state NULL");
  if (b->n > 0x7fffffffLL) return fail(BMADGPU_EINVAL, "more than 2^31-1 particles in one bunch");
  return BMADGPU_OK;
}

int check_range(const bmadgpu_lattice* lat, int32_t ix_start, int32_t ix_end, int32_t n_turns) {
  if (!lat) return fail(BMADGPU_EINVAL, "lattice is NULL");
  int n = (int)lat->pk.info.n_ele;
  if (ix_start < 0 || ix_end > n || ix_start >= ix_end) return fail(BMADGPU_EINVAL, "element range out of bounds");
  if (n_turns < 0) return fail(BMADGPU_EINVAL, "n_turns < 0");
  return BMADGPU_OK;
}

}  // namespace

namespace bmadgpu {

// Core device-side tracking: all bunch pointers are device pointers.
int track_device(bmadgpu_ctx* c, const bmadgpu_lattice* lat, const bmadgpu_bunch* b, int32_t ix_start,
                 int32_t ix_end, int32_t turn0, int32_t n_turns, double* d_moments) {
  if (b->n == 0 || n_turns == 0) return BMADGPU_OK;
  const bmadgpu_tuning& tu = c->tuning;
  int per_launch = tu.turns_per_launch > 0 ? tu.turns_per_launch : n_turns;
  bool compact = tu.compact && per_launch < n_turns;
  if (compact) {
    int r = ensure_live(c, b->n);
    if (r) return r;
  }
  if (d_moments) CUDA_TRY(cudaMemsetAsync(d_moments, 0, (size_t)n_turns * BMADGPU_N_MOMENTS * sizeof(double), c->stream));
  k_set_i64<<<1, 1, 0, c->stream>>>(c->d_nwork, b->n);
  CUDA_TRY(cudaGetLastError());
  c->launches++;
  TrackArgs a;
  std::memset(&a, 0, sizeof(a));
  a.table = lat->d_table;
  a.table_bytes = lat->pk.info.total_bytes;
  a.rare = (int32_t)lat->pk.info.rare;
  a.hdr_bytes = lat->pk.info.hdr_bytes;
  a.ap_bytes = lat->pk.info.ap_bytes;
  a.ix_start = ix_start;
  a.ix_end = ix_end;
  a.ld = b->n;
  a.vec = b->vec;
  a.beta = b->beta;
  a.t = b->t;
  a.state = b->state;
  a.ix_ele = b->ix_ele;
  a.ix_turn = b->ix_turn;
  a.location = b->location;
  a.ref_prefix = lat->d_prefix;
  a.G = lat->G;
  a.err_flag = c->d_err;
  LaunchCfg cfg;
  cfg.block = tu.block;
  cfg.ctas_per_sm = tu.ctas_per_sm;
  cfg.stage_smem = tu.stage_smem != 0;
  int cur = 0;  // which live list / count is current; live == nullptr means identity
  const int32_t* live = nullptr;
  for (int32_t done = 0; done < n_turns; done += per_launch) {
    int32_t nt = std::min(per_launch, n_turns - done);
    a.turn0 = turn0 + done;
    a.n_turns = nt;
    a.n_work = c->d_nwork + cur;
    a.live = live;
    a.moments = d_moments ? d_moments + (int64_t)done * BMADGPU_N_MOMENTS : nullptr;
    CUDA_TRY(launch_track(a, cfg, c->sm_count, c->stream));
    c->launches++;
    if (compact && done + nt < n_turns) {
      int nxt = live ? 1 - cur : 0;
      if (!live) nxt = 1;  // first compaction: identity list -> list 1
      CUDA_TRY(launch_compact(b->state, live, c->d_nwork + cur, b->n, c->d_live[nxt], c->d_nwork + nxt, c->stream));
      c->launches++;
      live = c->d_live[nxt];
      cur = nxt;
    }
  }
  return BMADGPU_OK;
}


Globals make_globals(const bmadgpu_param& p) {
  Globals g;
  g.p0c = p.p0c;
  g.e_tot = p.e_tot;
  g.mass = p.mass;
  g.beta0 = p.p0c / p.e_tot;
  g.max_ap = p.max_aperture_limit;
  g.mass2 = p.mass * p.mass;
  // low_energy_z_correction.f90:43-45 constants, same expressions
  double me = p.mass / p.e_tot;
  g.lez_me2 = me * me;
  g.lez_b02 = g.beta0 * g.beta0;
  g.lez_f = g.lez_b02 * (2 * g.lez_b02 - g.lez_me2 / 2);
  g.lez_thresh = 3e-7 * p.e_tot;
  g.charge = p.charge;
  g.inv_beta0 = 1 / g.beta0;
  return g;
}

int check_err_flag(bmadgpu_ctx* c) {
  int32_t h = 0;
  CUDA_TRY(cudaMemcpyAsync(&h, c->d_err, sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  if (h) {
    cudaMemsetAsync(c->d_err, 0, sizeof(int32_t), c->stream);
    return fail(BMADGPU_ETIMEDOUT, "element-table staging wait timed out (results used the global-memory table)");
  }
  return BMADGPU_OK;
}

int noalloc_fail(int code, const char* msg) { return fail(code, msg); }

// Argument checks and kernel arguments for bmadgpu_track_bunch_device_noalloc (noalloc.cu); makes
// the context's device current. Allocates nothing.
int noalloc_prepare(bmadgpu_ctx* c, const bmadgpu_lattice* lat, const bmadgpu_bunch* b, TrackArgs* a,
                    LaunchCfg* cfg, int* sm_count, cudaStream_t* stream, int64_t** launches) {
  if (!c) return fail(BMADGPU_EINVAL, "ctx is NULL");
  int r = check_bunch(b);
  if (r) return r;
  if ((r = check_range(lat, 0, (int32_t)(lat ? lat->pk.info.n_ele : 1), 0))) return r;
  if (lat->device != c->device) return fail(BMADGPU_EINVAL, "lattice and context are on different devices");
  CUDA_TRY(cudaSetDevice(c->device));
  std::memset(a, 0, sizeof(*a));
  a->table = lat->d_table;
  a->table_bytes = lat->pk.info.total_bytes;
  a->rare = (int32_t)lat->pk.info.rare;
  a->hdr_bytes = lat->pk.info.hdr_bytes;
  a->ap_bytes = lat->pk.info.ap_bytes;
  a->ix_start = 0;
  a->ix_end = (int32_t)lat->pk.info.n_ele;
  a->ld = b->n;
  a->vec = b->vec;
  a->beta = b->beta;
  a->t = b->t;
  a->state = b->state;
  a->ix_ele = b->ix_ele;
  a->ix_turn = b->ix_turn;
  a->location = b->location;
  a->ref_prefix = lat->d_prefix;
  a->G = lat->G;
  a->err_flag = c->d_err;
  cfg->block = c->tuning.block;
  cfg->ctas_per_sm = c->tuning.ctas_per_sm;
  cfg->stage_smem = c->tuning.stage_smem != 0;
  *sm_count = c->sm_count;
  *stream = c->stream;
  *launches = &c->launches;
  return BMADGPU_OK;
}

}  // namespace bmadgpu

extern "C" {

int bmadgpu_abi_version(void) { return BMADGPU_ABI_VERSION; }

const char* bmadgpu_last_error(void) { return g_last_error.c_str(); }

int64_t bmadgpu_sizeof(int32_t which) {
  switch (which) {
    case 0: return (int64_t)sizeof(bmadgpu_element);
    case 1: return (int64_t)sizeof(bmadgpu_param);
    case 2: return (int64_t)sizeof(bmadgpu_bunch);
    case 3: return (int64_t)sizeof(bmadgpu_tuning);
    case 4: return (int64_t)sizeof(bmadgpu_batch_tuning);
    case 5: return (int64_t)sizeof(bmadgpu_server_config);
    case 6: return (int64_t)sizeof(bmadgpu_job_info);
    case 7: return (int64_t)sizeof(bmadgpu_server_stats);
    case 8: return (int64_t)sizeof(bmadgpu_bunch_data);
    case 9: return (int64_t)sizeof(bmadgpu_ltt_params);
    case 10: return (int64_t)sizeof(bmadgpu_da_params);
    case 11: return (int64_t)sizeof(bmadgpu_da_point);
    case 12: return (int64_t)sizeof(bmadgpu_twiss);
    case 13: return (int64_t)sizeof(bmadgpu_beam_init);
    case 14: return (int64_t)sizeof(bmadgpu_fma_params);
    case 15: return (int64_t)sizeof(bmadgpu_fma_point);
  }
  return -1;
}

int bmadgpu_ctx_create(int32_t device, bmadgpu_ctx** out) {
  if (!out) return fail(BMADGPU_EINVAL, "out is NULL");
  *out = nullptr;
  int n_dev = 0;
  cudaError_t e = cudaGetDeviceCount(&n_dev);
  if (e != cudaSuccess || n_dev == 0) return fail(BMADGPU_ECUDA, "no CUDA device available");
  if (device < 0 || device >= n_dev) return fail(BMADGPU_EINVAL, "device index out of range");
  CUDA_TRY(cudaSetDevice(device));
  cudaDeviceProp prop;
  CUDA_TRY(cudaGetDeviceProperties(&prop, device));
  if (prop.major < 10) return fail(BMADGPU_EUNSUPPORTED, "needs an sm_100 (Blackwell B200) device");
  CUDA_TRY(upload_constants());
  bmadgpu_ctx* c = new (std::nothrow) bmadgpu_ctx();
  if (!c) return fail(BMADGPU_ENOMEM, "host allocation failed");
  c->device = device;
  c->sm_count = prop.multiProcessorCount;
  c->tuning = bmadgpu_tuning{256, 2, 1, 0, 0, {0, 0, 0}};
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc(&c->d_err, sizeof(int32_t)) != cudaSuccess ||
      cudaMalloc(&c->d_nwork, 2 * sizeof(int64_t)) != cudaSuccess) {
    bmadgpu_ctx_destroy(c);
    return fail(BMADGPU_ENOMEM, "cannot create stream or device scalars");
  }
  cudaMemset(c->d_err, 0, sizeof(int32_t));
  *out = c;
  return BMADGPU_OK;
}

int bmadgpu_ctx_destroy(bmadgpu_ctx* c) {
  if (!c) return BMADGPU_OK;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  cudaFree(c->d_err);
  cudaFree(c->d_nwork);
  cudaFree(c->d_live[0]);
  cudaFree(c->d_live[1]);
  cudaFree(c->d_vec);
  cudaFree(c->d_beta);
  cudaFree(c->d_t);
  cudaFree(c->d_i32);
  cudaFree(c->d_mom);
  cudaFree(c->d_tvec);
  cudaFree(c->d_tbeta);
  cudaFree(c->d_tstate);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return BMADGPU_OK;
}

int bmadgpu_ctx_synchronize(bmadgpu_ctx* c) {
  if (!c) return fail(BMADGPU_EINVAL, "ctx is NULL");
  CUDA_TRY(cudaSetDevice(c->device));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  return check_err_flag(c);
}

int64_t bmadgpu_ctx_launch_count(const bmadgpu_ctx* c) { return c ? c->launches : -1; }

int bmadgpu_measure_fp64_peak(bmadgpu_ctx* c, double* flops_per_s) {
  if (!c || !flops_per_s) return fail(BMADGPU_EINVAL, "NULL argument");
  CUDA_TRY(cudaSetDevice(c->device));
  CUDA_TRY(measure_fp64_peak(c->sm_count, c->stream, flops_per_s));
  c->launches += 2;
  return BMADGPU_OK;
}

int bmadgpu_ctx_set_tuning(bmadgpu_ctx* c, const bmadgpu_tuning* t) {
  if (!c || !t) return fail(BMADGPU_EINVAL, "NULL argument");
  if (t->block != 64 && t->block != 128 && t->block != 256 && t->block != 512)
    return fail(BMADGPU_EINVAL, "block must be 64, 128, 256 or 512");
  if (t->ctas_per_sm < 0 || t->turns_per_launch < 0) return fail(BMADGPU_EINVAL, "negative tuning value");
  c->tuning = *t;
  return BMADGPU_OK;
}

int bmadgpu_ctx_get_tuning(const bmadgpu_ctx* c, bmadgpu_tuning* t) {
  if (!c || !t) return fail(BMADGPU_EINVAL, "NULL argument");
  *t = c->tuning;
  return BMADGPU_OK;
}

int bmadgpu_ctx_info(const bmadgpu_ctx* c, int32_t* device, int32_t* sm_count, void** stream) {
  if (!c) return fail(BMADGPU_EINVAL, "ctx is NULL");
  if (device) *device = c->device;
  if (sm_count) *sm_count = c->sm_count;
  if (stream) *stream = (void*)c->stream;
  return BMADGPU_OK;
}

int bmadgpu_lattice_create(bmadgpu_ctx* c, const bmadgpu_element* eles, int32_t n_ele,
                           const bmadgpu_param* param, bmadgpu_lattice** out) {
  if (!c || !eles || !param || !out) return fail(BMADGPU_EINVAL, "NULL argument");
  *out = nullptr;
  bmadgpu_lattice* L = new (std::nothrow) bmadgpu_lattice();
  if (!L) return fail(BMADGPU_ENOMEM, "host allocation failed");
  std::string err;
  int r = pack_lattice(eles, n_ele, *param, L->pk, err);
  if (r) {
    delete L;
    return fail(r, err);
  }
  L->device = c->device;
  L->param = *param;
  L->eles.assign(eles, eles + n_ele);
  L->G = make_globals(*param);
  cudaSetDevice(c->device);
  size_t nb = L->pk.image.size();
  if (cudaMalloc(&L->d_table, nb) != cudaSuccess ||
      cudaMalloc(&L->d_prefix, L->pk.ref_time_prefix.size() * sizeof(double)) != cudaSuccess) {
    bmadgpu_lattice_destroy(L);
    return fail(BMADGPU_ENOMEM, "cannot allocate the device element table");
  }
  if (cudaMemcpy(L->d_table, L->pk.image.data(), nb, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(L->d_prefix, L->pk.ref_time_prefix.data(), L->pk.ref_time_prefix.size() * sizeof(double),
                 cudaMemcpyHostToDevice) != cudaSuccess) {
    bmadgpu_lattice_destroy(L);
    return fail(BMADGPU_ECUDA, "cannot upload the element table");
  }
  *out = L;
  return BMADGPU_OK;
}

int bmadgpu_lattice_check(const bmadgpu_element* eles, int32_t n_ele, const bmadgpu_param* param,
                          int32_t* n_step_out, int64_t* table_bytes) {
  if (!eles || !param) return fail(BMADGPU_EINVAL, "NULL argument");
  PackedLattice pk;
  std::string err;
  int r = pack_lattice(eles, n_ele, *param, pk, err);
  if (r) return fail(r, err);
  if (n_step_out)
    for (int32_t i = 0; i < n_ele; i++) n_step_out[i] = pk.n_step[i];
  if (table_bytes) *table_bytes = (int64_t)pk.info.total_bytes;
  return BMADGPU_OK;
}

int bmadgpu_lattice_destroy(bmadgpu_lattice* L) {
  if (!L) return BMADGPU_OK;
  cudaSetDevice(L->device);
  cudaFree(L->d_table);
  cudaFree(L->d_prefix);
  delete L;
  return BMADGPU_OK;
}

int32_t bmadgpu_lattice_n_step(const bmadgpu_lattice* L, int32_t i) {
  if (!L || i < 0 || i >= (int32_t)L->pk.n_step.size()) return -1;
  return L->pk.n_step[i];
}

int64_t bmadgpu_lattice_table_bytes(const bmadgpu_lattice* L) {
  if (!L) return -1;
  return (int64_t)L->pk.info.total_bytes;
}

int bmadgpu_track_bunch_device(bmadgpu_ctx* c, const bmadgpu_lattice* lat, bmadgpu_bunch* b, int32_t ix_start,
                               int32_t ix_end, int32_t turn0, int32_t n_turns, double* moments) {
  if (!c) return fail(BMADGPU_EINVAL, "ctx is NULL");
  int r = check_bunch(b);
  if (r) return r;
  if ((r = check_range(lat, ix_start, ix_end, n_turns))) return r;
  if (lat->device != c->device) return fail(BMADGPU_EINVAL, "lattice and context are on different devices");
  CUDA_TRY(cudaSetDevice(c->device));
  return track_device(c, lat, b, ix_start, ix_end, turn0, n_turns, moments);
}

int bmadgpu_track_bunch(bmadgpu_ctx* c, const bmadgpu_lattice* lat, bmadgpu_bunch* b, int32_t ix_start,
                        int32_t ix_end, int32_t turn0, int32_t n_turns, double* moments) {
  if (!c) return fail(BMADGPU_EINVAL, "ctx is NULL");
  int r = check_bunch(b);
  if (r) return r;
  if ((r = check_range(lat, ix_start, ix_end, n_turns))) return r;
  if (lat->device != c->device) return fail(BMADGPU_EINVAL, "lattice and context are on different devices");
  CUDA_TRY(cudaSetDevice(c->device));
  const int64_t n = b->n;
  if (n == 0 || n_turns == 0) return BMADGPU_OK;
  if ((r = ensure_staging(c, n))) return r;
  if (moments && (int64_t)n_turns * BMADGPU_N_MOMENTS > c->mom_cap) {
    cudaFree(c->d_mom);
    c->d_mom = nullptr;
    c->mom_cap = 0;
    if (cudaMalloc(&c->d_mom, (size_t)n_turns * BMADGPU_N_MOMENTS * sizeof(double)) != cudaSuccess)
      return fail(BMADGPU_ENOMEM, "cannot allocate the moments buffer");
    c->mom_cap = (int64_t)n_turns * BMADGPU_N_MOMENTS;
  }
  cudaStream_t s = c->stream;
  bmadgpu_bunch d;
  d.n = n;
  d.vec = c->d_vec;
  d.beta = c->d_beta;
  d.t = b->t ? c->d_t : nullptr;
  d.state = c->d_i32;
  d.ix_ele = b->ix_ele ? c->d_i32 + n : nullptr;
  d.ix_turn = b->ix_turn ? c->d_i32 + 2 * n : nullptr;
  d.location = b->location ? c->d_i32 + 3 * n : nullptr;
  const size_t nd = (size_t)n * sizeof(double), ni = (size_t)n * sizeof(int32_t);
  CUDA_TRY(cudaMemcpyAsync(d.vec, b->vec, 6 * nd, cudaMemcpyHostToDevice, s));
  CUDA_TRY(cudaMemcpyAsync(d.beta, b->beta, nd, cudaMemcpyHostToDevice, s));
  if (d.t) CUDA_TRY(cudaMemcpyAsync(d.t, b->t, nd, cudaMemcpyHostToDevice, s));
  CUDA_TRY(cudaMemcpyAsync(d.state, b->state, ni, cudaMemcpyHostToDevice, s));
  if (d.ix_ele) CUDA_TRY(cudaMemcpyAsync(d.ix_ele, b->ix_ele, ni, cudaMemcpyHostToDevice, s));
  if (d.ix_turn) CUDA_TRY(cudaMemcpyAsync(d.ix_turn, b->ix_turn, ni, cudaMemcpyHostToDevice, s));
  if (d.location) CUDA_TRY(cudaMemcpyAsync(d.location, b->location, ni, cudaMemcpyHostToDevice, s));
  if ((r = track_device(c, lat, &d, ix_start, ix_end, turn0, n_turns, moments ? c->d_mom : nullptr))) return r;
  CUDA_TRY(cudaMemcpyAsync(b->vec, d.vec, 6 * nd, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaMemcpyAsync(b->beta, d.beta, nd, cudaMemcpyDeviceToHost, s));
  if (d.t) CUDA_TRY(cudaMemcpyAsync(b->t, d.t, nd, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaMemcpyAsync(b->state, d.state, ni, cudaMemcpyDeviceToHost, s));
  if (d.ix_ele) CUDA_TRY(cudaMemcpyAsync(b->ix_ele, d.ix_ele, ni, cudaMemcpyDeviceToHost, s));
  if (d.ix_turn) CUDA_TRY(cudaMemcpyAsync(b->ix_turn, d.ix_turn, ni, cudaMemcpyDeviceToHost, s));
  if (d.location) CUDA_TRY(cudaMemcpyAsync(b->location, d.location, ni, cudaMemcpyDeviceToHost, s));
  if (moments)
    CUDA_TRY(cudaMemcpyAsync(moments, c->d_mom, (size_t)n_turns * BMADGPU_N_MOMENTS * sizeof(double),
                             cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  return check_err_flag(c);
}

int bmadgpu_autotune(bmadgpu_ctx* c, const bmadgpu_lattice* lat, const bmadgpu_bunch* b, int64_t sample_n,
                     bmadgpu_tuning* chosen) {
  if (!c || !lat || !b) return fail(BMADGPU_EINVAL, "NULL argument");
  int r = check_bunch(b);
  if (r) return r;
  CUDA_TRY(cudaSetDevice(c->device));
  // Trials on up to 8192 particles per SM (the whole bunch of a 1M-particle run): shapes that tie on
  // a few waves of particles can differ by 10 % over many waves.
  int64_t m = std::min<int64_t>(b->n, sample_n > 0 ? sample_n : (int64_t)c->sm_count * 8192);
  if (m <= 0) return fail(BMADGPU_EINVAL, "empty bunch");
  if (m > c->tune_cap) {
    cudaFree(c->d_tvec);
    cudaFree(c->d_tbeta);
    cudaFree(c->d_tstate);
    c->d_tvec = nullptr; c->d_tbeta = nullptr; c->d_tstate = nullptr;
    c->tune_cap = 0;
    if (cudaMalloc(&c->d_tvec, (size_t)m * 6 * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&c->d_tbeta, (size_t)m * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&c->d_tstate, (size_t)m * sizeof(int32_t)) != cudaSuccess)
      return fail(BMADGPU_ENOMEM, "cannot allocate autotuner trial buffers");
    c->tune_cap = m;
  }
  bmadgpu_bunch t;
  std::memset(&t, 0, sizeof(t));
  t.n = m;
  t.vec = c->d_tvec;
  t.beta = c->d_tbeta;
  t.state = c->d_tstate;
  const bmadgpu_tuning saved = c->tuning;
  struct Cand { int block, ctas, stage; };
  static const Cand cands[] = {{128, 0, 0}, {128, 4, 0}, {128, 5, 0}, {128, 6, 0}, {256, 0, 0}, {256, 2, 0},
                               {256, 3, 0}, {64, 8, 0},  {64, 12, 0}, {128, 0, 1}, {128, 4, 1}, {256, 2, 1}};
  cudaEvent_t e0, e1;
  CUDA_TRY(cudaEventCreate(&e0));
  CUDA_TRY(cudaEventCreate(&e1));
  float best_ms = 1e30f;
  bmadgpu_tuning best = saved;
  for (const Cand& k : cands) {
    if (k.stage && !table_fits_smem(lat->pk.info.total_bytes)) continue;
    CUDA_TRY(cudaMemcpy2DAsync(t.vec, m * sizeof(double), b->vec, b->n * sizeof(double), m * sizeof(double), 6,
                               cudaMemcpyDeviceToDevice, c->stream));
    CUDA_TRY(cudaMemcpyAsync(t.beta, b->beta, m * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    CUDA_TRY(cudaMemcpyAsync(t.state, b->state, m * sizeof(int32_t), cudaMemcpyDeviceToDevice, c->stream));
    c->tuning = bmadgpu_tuning{k.block, k.ctas, k.stage, 0, 0, {0, 0, 0}};
    CUDA_TRY(cudaEventRecord(e0, c->stream));
    r = track_device(c, lat, &t, 0, (int32_t)lat->pk.info.n_ele, 0, 1, nullptr);
    CUDA_TRY(cudaEventRecord(e1, c->stream));
    if (r) {
      c->tuning = saved;
      return r;
    }
    CUDA_TRY(cudaEventSynchronize(e1));
    float ms = 0;
    CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
    // a second turn of the same particles: the shorter of the two timings counts
    CUDA_TRY(cudaEventRecord(e0, c->stream));
    r = track_device(c, lat, &t, 0, (int32_t)lat->pk.info.n_ele, 1, 1, nullptr);
    CUDA_TRY(cudaEventRecord(e1, c->stream));
    if (r) {
      c->tuning = saved;
      return r;
    }
    CUDA_TRY(cudaEventSynchronize(e1));
    float ms2 = 0;
    CUDA_TRY(cudaEventElapsedTime(&ms2, e0, e1));
    ms = std::min(ms, ms2);
    if (ms < best_ms) {
      best_ms = ms;
      best = c->tuning;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  best.turns_per_launch = saved.turns_per_launch;
  best.compact = saved.compact;
  c->tuning = best;
  if (chosen) *chosen = best;
  return check_err_flag(c);
}

int bmadgpu_track1_bunch(bmadgpu_ctx* c, const bmadgpu_lattice* lat, bmadgpu_bunch* b, int32_t ix_ele,
                         int32_t turn) {
  return bmadgpu_track_bunch(c, lat, b, ix_ele, ix_ele + 1, turn, 1, nullptr);
}

}  // extern "C"
