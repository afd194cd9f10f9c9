// batch_capi.cu -- extern "C" batch entry points of include/bmadgpu.h.
//
// A batch owns the device particle state of all its variants, the per-variant descriptors, two
// live-index lists with their per-variant lengths, the work plan (tile prefix) and the work-item
// counter. A call enqueues: set per-variant turns, then plan -> track [-> plan -> track ...] with
// one track launch per turns_per_launch turns. With use_graph the plan/track sequence is captured
// once per (n_turns, tuning) into a CUDA graph and replayed; the per-call turn numbers are written
// by a kernel launched before the graph, so the graph itself never changes.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <new>
#include <vector>

#include "batch.cuh"
#include "capi_internal.h"

using namespace bmadgpu;

struct bmadgpu_batch {
  bmadgpu_ctx* ctx = nullptr;
  int32_t n_var = 0;
  int64_t total = 0;
  std::vector<int64_t> counts, offs;
  BatchVar* d_vars = nullptr;
  double* d_vec = nullptr;        // [6 * total]
  double* d_beta = nullptr;       // [total]
  double* d_t = nullptr;          // [total]
  int32_t* d_i32 = nullptr;       // state, ix_ele, ix_turn, location: [4 * total]
  int32_t* d_live[2] = {nullptr, nullptr};
  unsigned long long* d_cnt = nullptr;  // [2 * n_var]
  int64_t* d_prefix = nullptr;          // [n_var + 1]
  unsigned long long* d_queue = nullptr;
  uint32_t smem_bytes = 0;        // largest stageable table
  int32_t rare = 0;               // some variant's table has extra blocks / pitched offsets
  bmadgpu_batch_tuning tuning;
  cudaGraphExec_t exec = nullptr;
  int32_t graph_turns = -1;
  bmadgpu_batch_tuning graph_tuning;
  int64_t graph_launches = 0;     // kernel launches in the captured graph
  unsigned char* d_save = nullptr;  // autotuner copy of the particle state
};

namespace {

constexpr uint32_t kMaxStageBytes = 200 * 1024;

size_t state_bytes(int64_t total) { return (size_t)total * (8 * sizeof(double) + 4 * sizeof(int32_t)); }

bool same_tuning(const bmadgpu_batch_tuning& a, const bmadgpu_batch_tuning& b) {
  return a.block == b.block && a.ctas_per_sm == b.ctas_per_sm && a.particles_per_thread == b.particles_per_thread &&
         a.turns_per_launch == b.turns_per_launch && a.stage_smem == b.stage_smem;
}

int check_tuning(const bmadgpu_batch_tuning* t) {
  if (t->block != 64 && t->block != 128 && t->block != 256 && t->block != 512)
    return fail(BMADGPU_EINVAL, "block must be 64, 128, 256 or 512");
  if (t->ctas_per_sm < 0 || t->turns_per_launch < 0) return fail(BMADGPU_EINVAL, "negative tuning value");
  if (t->particles_per_thread < 1 || t->particles_per_thread > 64)
    return fail(BMADGPU_EINVAL, "particles_per_thread must be 1 .. 64");
  return BMADGPU_OK;
}

void drop_graph(bmadgpu_batch* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  b->exec = nullptr;
  b->graph_turns = -1;
}

// Kernel and grid of the batch's current tuning (function attributes are set here, never
// during stream capture).
int resolve(bmadgpu_batch* b, BatchKernel* k) {
  const bmadgpu_batch_tuning& tu = b->tuning;
  BatchLaunch cfg;
  cfg.block = tu.block;
  cfg.ctas_per_sm = tu.ctas_per_sm;
  cfg.particles_per_thread = tu.particles_per_thread;
  CUDA_TRY(batch_resolve(cfg, tu.stage_smem ? b->smem_bytes : 0, b->ctx->sm_count, k));
  return BMADGPU_OK;
}

// Enqueues the plan/track sequence of one call (n_turns > 0) on the context stream.
int enqueue_calls(bmadgpu_batch* b, const BatchKernel& k, int32_t n_turns, int64_t* launches) {
  const bmadgpu_batch_tuning& tu = b->tuning;
  const uint32_t smem = k.smem;
  const int32_t tile = tu.block * tu.particles_per_thread;
  const int32_t tpl = tu.turns_per_launch > 0 ? std::min(tu.turns_per_launch, n_turns) : n_turns;
  const int32_t n_chunks = (n_turns + tpl - 1) / tpl;
  cudaStream_t s = b->ctx->stream;
  CUDA_TRY(batch_launch_plan(b->d_vars, b->n_var, tile, 0, true, nullptr, b->d_prefix, b->d_queue, b->d_cnt, s));
  (*launches)++;
  BatchArgs a;
  std::memset(&a, 0, sizeof(a));
  a.vars = b->d_vars;
  a.n_var = b->n_var;
  a.tile = tile;
  a.vec = b->d_vec;
  a.beta = b->d_beta;
  a.t = b->d_t;
  a.state = b->d_i32;
  a.ix_ele = b->d_i32 + b->total;
  a.ix_turn = b->d_i32 + 2 * b->total;
  a.location = b->d_i32 + 3 * b->total;
  a.tile_prefix = b->d_prefix;
  a.queue = b->d_queue;
  a.err_flag = b->ctx->d_err;
  a.smem_bytes = smem;
  a.rare = b->rare;
  for (int32_t c = 0; c < n_chunks; ++c) {
    const bool last = c == n_chunks - 1;
    a.turn_off = c * tpl;
    a.n_turns = std::min(tpl, n_turns - c * tpl);
    a.live_in = c == 0 ? nullptr : b->d_live[(c - 1) & 1];
    a.n_in = c == 0 ? nullptr : b->d_cnt + (size_t)((c - 1) & 1) * b->n_var;
    a.live_out = last ? nullptr : b->d_live[c & 1];
    a.n_out = last ? nullptr : b->d_cnt + (size_t)(c & 1) * b->n_var;
    CUDA_TRY(batch_launch_track(k, a, s));
    (*launches)++;
    if (!last) {
      CUDA_TRY(batch_launch_plan(b->d_vars, b->n_var, tile, (c + 1) * tpl, false, a.n_out, b->d_prefix, b->d_queue,
                                 b->d_cnt + (size_t)((c + 1) & 1) * b->n_var, s));
      (*launches)++;
    }
  }
  return BMADGPU_OK;
}

int track_call(bmadgpu_batch* b, int32_t turn0, int32_t n_turns, bool allow_graph) {
  bmadgpu_ctx* c = b->ctx;
  if (n_turns == 0 || b->total == 0) return BMADGPU_OK;
  BatchKernel k;
  int r = resolve(b, &k);
  if (r) return r;
  CUDA_TRY(batch_launch_set_turns(b->d_vars, b->n_var, turn0, n_turns, c->stream));
  c->launches++;
  if (!(allow_graph && b->tuning.use_graph)) {
    int64_t n = 0;
    r = enqueue_calls(b, k, n_turns, &n);
    c->launches += n;
    return r;
  }
  if (!b->exec || b->graph_turns != n_turns || !same_tuning(b->graph_tuning, b->tuning)) {
    drop_graph(b);
    int64_t n = 0;
    CUDA_TRY(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    r = enqueue_calls(b, k, n_turns, &n);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(c->stream, &g);
    if (r) {
      if (g) cudaGraphDestroy(g);
      return r;
    }
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
    e = cudaGraphInstantiate(&b->exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
      b->exec = nullptr;
      return cuda_fail(e, "cudaGraphInstantiate");
    }
    b->graph_turns = n_turns;
    b->graph_tuning = b->tuning;
    b->graph_launches = n;
  }
  CUDA_TRY(cudaGraphLaunch(b->exec, c->stream));
  c->launches += b->graph_launches;
  return BMADGPU_OK;
}

// Byte ranges of variant v (or of everything for v = -1) in the batch arrays.
struct Range {
  int64_t off, n;
};

int range_of(const bmadgpu_batch* b, int32_t v, Range* r) {
  if (v == -1) {
    r->off = 0;
    r->n = b->total;
    return BMADGPU_OK;
  }
  if (v < 0 || v >= b->n_var) return fail(BMADGPU_EINVAL, "variant index out of range");
  r->off = b->offs[v];
  r->n = b->counts[v];
  return BMADGPU_OK;
}

}  // namespace

extern "C" {

int bmadgpu_batch_create(bmadgpu_ctx* c, int32_t n_var, const bmadgpu_lattice* const* lats, const int64_t* counts,
                         bmadgpu_batch** out) {
  if (!c || !out || (n_var > 0 && (!lats || !counts))) return fail(BMADGPU_EINVAL, "NULL argument");
  *out = nullptr;
  if (n_var < 1) return fail(BMADGPU_EINVAL, "a batch needs at least one variant");
  int64_t total = 0;
  for (int32_t v = 0; v < n_var; ++v) {
    if (!lats[v]) return fail(BMADGPU_EINVAL, "lattice is NULL");
    if (lats[v]->device != c->device) return fail(BMADGPU_EINVAL, "lattice and context are on different devices");
    if (counts[v] < 0) return fail(BMADGPU_EINVAL, "negative particle count");
    total += counts[v];
  }
  if (total > 0x7fffffffLL) return fail(BMADGPU_EINVAL, "more than 2^31-1 particles in one batch");
  CUDA_TRY(cudaSetDevice(c->device));
  bmadgpu_batch* b = new (std::nothrow) bmadgpu_batch();
  if (!b) return fail(BMADGPU_ENOMEM, "host allocation failed");
  b->ctx = c;
  b->n_var = n_var;
  b->total = total;
  b->counts.assign(counts, counts + n_var);
  b->offs.resize(n_var);
  std::vector<BatchVar> hv(n_var);
  int64_t off = 0;
  for (int32_t v = 0; v < n_var; ++v) {
    const bmadgpu_lattice* L = lats[v];
    if (L->pk.info.rare) b->rare = 1;
    b->offs[v] = off;
    BatchVar& d = hv[v];
    std::memset(&d, 0, sizeof(d));
    d.table = L->d_table;
    d.ref_prefix = L->d_prefix;
    d.n = counts[v];
    d.off = off;
    d.table_bytes = L->pk.info.total_bytes;
    d.hdr_bytes = L->pk.info.hdr_bytes;
    d.ap_bytes = L->pk.info.ap_bytes;
    d.n_ele = L->pk.info.n_ele;
    d.G = L->G;
    if (d.table_bytes <= kMaxStageBytes) b->smem_bytes = std::max(b->smem_bytes, d.table_bytes);
    off += counts[v];
  }
  const size_t T = (size_t)std::max<int64_t>(total, 1);
  b->tuning = bmadgpu_batch_tuning{128, 0, 1, 0, 1, 1, {0, 0}};
  if (cudaMalloc(&b->d_vars, sizeof(BatchVar) * n_var) != cudaSuccess ||
      cudaMalloc(&b->d_vec, 6 * T * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&b->d_beta, T * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&b->d_t, T * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&b->d_i32, 4 * T * sizeof(int32_t)) != cudaSuccess ||
      cudaMalloc(&b->d_live[0], T * sizeof(int32_t)) != cudaSuccess ||
      cudaMalloc(&b->d_live[1], T * sizeof(int32_t)) != cudaSuccess ||
      cudaMalloc(&b->d_cnt, 2 * sizeof(unsigned long long) * n_var) != cudaSuccess ||
      cudaMalloc(&b->d_prefix, sizeof(int64_t) * (n_var + 1)) != cudaSuccess ||
      cudaMalloc(&b->d_queue, sizeof(unsigned long long)) != cudaSuccess) {
    bmadgpu_batch_destroy(b);
    return fail(BMADGPU_ENOMEM, "cannot allocate the batch's device state");
  }
  cudaStream_t s = c->stream;
  if (cudaMemcpyAsync(b->d_vars, hv.data(), sizeof(BatchVar) * n_var, cudaMemcpyHostToDevice, s) != cudaSuccess ||
      cudaMemsetAsync(b->d_vec, 0, 6 * T * sizeof(double), s) != cudaSuccess ||
      cudaMemsetAsync(b->d_beta, 0, T * sizeof(double), s) != cudaSuccess ||
      cudaMemsetAsync(b->d_t, 0, T * sizeof(double), s) != cudaSuccess ||
      cudaMemsetAsync(b->d_i32, 0, 4 * T * sizeof(int32_t), s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess) {
    bmadgpu_batch_destroy(b);
    return fail(BMADGPU_ECUDA, "cannot initialise the batch's device state");
  }
  *out = b;
  return BMADGPU_OK;
}

int bmadgpu_batch_destroy(bmadgpu_batch* b) {
  if (!b) return BMADGPU_OK;
  cudaSetDevice(b->ctx->device);
  cudaStreamSynchronize(b->ctx->stream);
  drop_graph(b);
  cudaFree(b->d_vars);
  cudaFree(b->d_vec);
  cudaFree(b->d_beta);
  cudaFree(b->d_t);
  cudaFree(b->d_i32);
  cudaFree(b->d_live[0]);
  cudaFree(b->d_live[1]);
  cudaFree(b->d_cnt);
  cudaFree(b->d_prefix);
  cudaFree(b->d_queue);
  cudaFree(b->d_save);
  delete b;
  return BMADGPU_OK;
}

int bmadgpu_batch_view(const bmadgpu_batch* b, int32_t v, bmadgpu_bunch* d) {
  if (!b || !d) return fail(BMADGPU_EINVAL, "NULL argument");
  Range r;
  int e = range_of(b, v, &r);
  if (e) return e;
  d->n = r.n;
  d->vec = b->d_vec + 6 * r.off;
  d->beta = b->d_beta + r.off;
  d->t = b->d_t + r.off;
  d->state = b->d_i32 + r.off;
  d->ix_ele = b->d_i32 + b->total + r.off;
  d->ix_turn = b->d_i32 + 2 * b->total + r.off;
  d->location = b->d_i32 + 3 * b->total + r.off;
  return BMADGPU_OK;
}

int bmadgpu_batch_upload(bmadgpu_batch* b, int32_t v, const bmadgpu_bunch* h) {
  if (!b || !h) return fail(BMADGPU_EINVAL, "NULL argument");
  bmadgpu_bunch d;
  int e = bmadgpu_batch_view(b, v, &d);
  if (e) return e;
  if (h->n != d.n) return fail(BMADGPU_EINVAL, "host bunch size differs from the variant's particle count");
  if (d.n == 0) return BMADGPU_OK;
  if (!h->vec || !h->beta || !h->state) return fail(BMADGPU_EINVAL, "bunch vec/beta/state NULL");
  CUDA_TRY(cudaSetDevice(b->ctx->device));
  cudaStream_t s = b->ctx->stream;
  const size_t nd = (size_t)d.n * sizeof(double), ni = (size_t)d.n * sizeof(int32_t);
  CUDA_TRY(cudaMemcpyAsync(d.vec, h->vec, 6 * nd, cudaMemcpyHostToDevice, s));
  CUDA_TRY(cudaMemcpyAsync(d.beta, h->beta, nd, cudaMemcpyHostToDevice, s));
  CUDA_TRY(cudaMemcpyAsync(d.state, h->state, ni, cudaMemcpyHostToDevice, s));
  if (h->t) CUDA_TRY(cudaMemcpyAsync(d.t, h->t, nd, cudaMemcpyHostToDevice, s));
  if (h->ix_ele) CUDA_TRY(cudaMemcpyAsync(d.ix_ele, h->ix_ele, ni, cudaMemcpyHostToDevice, s));
  if (h->ix_turn) CUDA_TRY(cudaMemcpyAsync(d.ix_turn, h->ix_turn, ni, cudaMemcpyHostToDevice, s));
  if (h->location) CUDA_TRY(cudaMemcpyAsync(d.location, h->location, ni, cudaMemcpyHostToDevice, s));
  return BMADGPU_OK;
}

int bmadgpu_batch_download(bmadgpu_batch* b, int32_t v, bmadgpu_bunch* h) {
  if (!b || !h) return fail(BMADGPU_EINVAL, "NULL argument");
  bmadgpu_bunch d;
  int e = bmadgpu_batch_view(b, v, &d);
  if (e) return e;
  if (h->n != d.n) return fail(BMADGPU_EINVAL, "host bunch size differs from the variant's particle count");
  CUDA_TRY(cudaSetDevice(b->ctx->device));
  cudaStream_t s = b->ctx->stream;
  if (d.n > 0) {
    if (!h->vec || !h->beta || !h->state) return fail(BMADGPU_EINVAL, "bunch vec/beta/state NULL");
    const size_t nd = (size_t)d.n * sizeof(double), ni = (size_t)d.n * sizeof(int32_t);
    CUDA_TRY(cudaMemcpyAsync(h->vec, d.vec, 6 * nd, cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaMemcpyAsync(h->beta, d.beta, nd, cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaMemcpyAsync(h->state, d.state, ni, cudaMemcpyDeviceToHost, s));
    if (h->t) CUDA_TRY(cudaMemcpyAsync(h->t, d.t, nd, cudaMemcpyDeviceToHost, s));
    if (h->ix_ele) CUDA_TRY(cudaMemcpyAsync(h->ix_ele, d.ix_ele, ni, cudaMemcpyDeviceToHost, s));
    if (h->ix_turn) CUDA_TRY(cudaMemcpyAsync(h->ix_turn, d.ix_turn, ni, cudaMemcpyDeviceToHost, s));
    if (h->location) CUDA_TRY(cudaMemcpyAsync(h->location, d.location, ni, cudaMemcpyDeviceToHost, s));
  }
  return check_err_flag(b->ctx);
}

int bmadgpu_batch_track(bmadgpu_batch* b, int32_t turn0, int32_t n_turns) {
  if (!b) return fail(BMADGPU_EINVAL, "batch is NULL");
  if (n_turns < 0) return fail(BMADGPU_EINVAL, "n_turns < 0");
  CUDA_TRY(cudaSetDevice(b->ctx->device));
  return track_call(b, turn0, n_turns, true);
}

int bmadgpu_batch_set_tuning(bmadgpu_batch* b, const bmadgpu_batch_tuning* t) {
  if (!b || !t) return fail(BMADGPU_EINVAL, "NULL argument");
  int r = check_tuning(t);
  if (r) return r;
  b->tuning = *t;
  return BMADGPU_OK;
}

int bmadgpu_batch_get_tuning(const bmadgpu_batch* b, bmadgpu_batch_tuning* t) {
  if (!b || !t) return fail(BMADGPU_EINVAL, "NULL argument");
  *t = b->tuning;
  return BMADGPU_OK;
}

int bmadgpu_batch_autotune(bmadgpu_batch* b, int32_t sample_turns, bmadgpu_batch_tuning* chosen) {
  if (!b) return fail(BMADGPU_EINVAL, "batch is NULL");
  if (sample_turns < 0) return fail(BMADGPU_EINVAL, "sample_turns < 0");
  if (sample_turns == 0) sample_turns = 8;
  bmadgpu_ctx* c = b->ctx;
  CUDA_TRY(cudaSetDevice(c->device));
  if (b->total == 0) {
    if (chosen) *chosen = b->tuning;
    return BMADGPU_OK;
  }
  const size_t sb = state_bytes(b->total);
  if (!b->d_save && cudaMalloc(&b->d_save, sb) != cudaSuccess) {
    b->d_save = nullptr;
    return fail(BMADGPU_ENOMEM, "cannot allocate the autotuner's state copy");
  }
  // The state arrays are four separate allocations; save and restore them one by one.
  const size_t T = (size_t)b->total;
  struct Piece {
    void* p;
    size_t bytes;
  } pieces[] = {{b->d_vec, 6 * T * sizeof(double)},
                {b->d_beta, T * sizeof(double)},
                {b->d_t, T * sizeof(double)},
                {b->d_i32, 4 * T * sizeof(int32_t)}};
  cudaStream_t s = c->stream;
  size_t at = 0;
  for (const Piece& p : pieces) {
    CUDA_TRY(cudaMemcpyAsync(b->d_save + at, p.p, p.bytes, cudaMemcpyDeviceToDevice, s));
    at += p.bytes;
  }
  cudaEvent_t e0, e1;
  CUDA_TRY(cudaEventCreate(&e0));
  CUDA_TRY(cudaEventCreate(&e1));
  const bmadgpu_batch_tuning saved = b->tuning;
  auto trial = [&](const bmadgpu_batch_tuning& t, int32_t turns, float* ms) -> int {
    b->tuning = t;
    size_t o = 0;
    for (const Piece& p : pieces) {
      CUDA_TRY(cudaMemcpyAsync(p.p, b->d_save + o, p.bytes, cudaMemcpyDeviceToDevice, s));
      o += p.bytes;
    }
    CUDA_TRY(cudaEventRecord(e0, s));
    int r = track_call(b, 0, turns, false);
    if (r) return r;
    CUDA_TRY(cudaEventRecord(e1, s));
    CUDA_TRY(cudaEventSynchronize(e1));
    CUDA_TRY(cudaEventElapsedTime(ms, e0, e1));
    return BMADGPU_OK;
  };
  int r = BMADGPU_OK;
  bmadgpu_batch_tuning best = saved;
  float best_ms = 1e30f;
  const int32_t short_turns = std::min<int32_t>(sample_turns, 4);
  // 1) launch shape (threads per CTA x register budget) and table staging
  struct Shape {
    int block, ctas;
  };
  static const Shape shapes[] = {{128, 0}, {128, 4}, {128, 5}, {128, 6}, {256, 0},
                                 {256, 2}, {256, 3}, {64, 8},  {64, 12}, {512, 1}};
  for (int stage = 1; stage >= 0 && !r; --stage) {
    if (stage && b->smem_bytes == 0) continue;
    for (const Shape& sh : shapes) {
      bmadgpu_batch_tuning t = saved;
      t.block = sh.block;
      t.ctas_per_sm = sh.ctas;
      t.particles_per_thread = 1;
      t.turns_per_launch = 0;
      t.stage_smem = stage;
      float ms = 0;
      if ((r = trial(t, short_turns, &ms))) break;
      if (ms < best_ms) {
        best_ms = ms;
        best = t;
      }
    }
  }
  // 2) particles per thread (work-item size)
  for (int ppt : {2, 4}) {
    if (r) break;
    bmadgpu_batch_tuning t = best;
    t.particles_per_thread = ppt;
    float ms = 0;
    if ((r = trial(t, short_turns, &ms))) break;
    if (ms < best_ms) {
      best_ms = ms;
      best = t;
    }
  }
  // 3) turns per launch (compaction interval), on sample_turns-turn trials
  if (!r) {
    best_ms = 1e30f;
    bmadgpu_batch_tuning best3 = best;
    int32_t last = -1;
    for (int div : {8, 4, 2, 1}) {
      const int32_t tpl = std::max<int32_t>(1, sample_turns / div);
      if (tpl == last) continue;
      last = tpl;
      bmadgpu_batch_tuning t = best;
      t.turns_per_launch = tpl;
      float ms = 0;
      if ((r = trial(t, sample_turns, &ms))) break;
      if (ms < best_ms) {
        best_ms = ms;
        best3 = t;
      }
    }
    best = best3;
  }
  // restore the state and keep the caller's graph setting
  size_t o = 0;
  for (const Piece& p : pieces) {
    cudaMemcpyAsync(p.p, b->d_save + o, p.bytes, cudaMemcpyDeviceToDevice, s);
    o += p.bytes;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (r) {
    b->tuning = saved;
    return r;
  }
  best.use_graph = saved.use_graph;
  b->tuning = best;
  if (chosen) *chosen = best;
  return check_err_flag(c);
}

}  // extern "C"
