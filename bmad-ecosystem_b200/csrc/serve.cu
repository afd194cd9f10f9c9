// serve.cu -- continuous-batching tracking server (bmadgpu_server_* of include/bmadgpu.h).
//
// Device side: one resident arena of particle state (the batched kernel's batch-wide arrays:
// vec [6][C], beta, t, state, ix_ele, ix_turn, location [C], two live lists [C]), the job-slot
// descriptors (BatchVar [max_jobs]) and the per-slot live counts (two sets). A job owns a slot and
// the particle range [off, off + n) of every arena array.
//
// Worker thread (the only thread that calls CUDA for the server):
//   admit   -- queued jobs in policy order while a slot, arena space and the live target allow;
//              their particles are copied in on the copy stream (overlapping the running round)
//              and their first live list is written on the compute stream;
//   round   -- descriptors for the round (turn0, turns) copied from a pinned mirror, then the
//              plan kernel and one k_batch_track launch over every resident job, then the new
//              live counts copied to pinned memory; at most two rounds are in flight;
//   retire  -- after a round completes, jobs whose turns are done or whose particles are all
//              lost are copied back on the copy stream (after the round's event), their slot and
//              arena range are released, and they are marked done when the copy's event fires.
// Ordering: every write to a job's arena range is on the copy stream (uploads, in admission
// order after the previous occupant's download) or in a round in which the job has work; a job
// being retired has no work in the rounds still in flight (its turns for them are zero or its
// live count is zero), so its range is never touched by a kernel while it is copied out or
// re-used.

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "batch.cuh"
#include "capi_internal.h"

using namespace bmadgpu;

namespace {

constexpr size_t kBytesPerParticle = 8 * sizeof(double) + 4 * sizeof(int32_t) + 2 * sizeof(int32_t);
constexpr uint32_t kServeStageBytes = 64 * 1024;
constexpr int kRoundsInFlight = 2;
constexpr size_t kMaxQueued = 1 << 20;
constexpr int kRecPar = 48;  // norm [36], closed orbit [6], z_limit, padding

// Record-arena layout of a frequency-map job of n particles and T turns (in doubles): the record
// [6][T][n], the parameters, the tunes [n][6], rec_state [2n] (int32) and fstate [n] (int32).
int64_t rec_doubles(int64_t n, int64_t T) { return 6 * T * n + kRecPar + 6 * n + n + n; }

double now_s() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

// First-fit allocator of particle ranges in [0, capacity) with coalescing.
class RangeAlloc {
 public:
  void reset(int64_t cap) {
    free_.clear();
    if (cap > 0) free_[0] = cap;
    used_ = 0;
  }
  int64_t alloc(int64_t n) {
    if (n <= 0) return 0;
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second >= n) {
        const int64_t off = it->first, len = it->second;
        free_.erase(it);
        if (len > n) free_[off + n] = len - n;
        used_ += n;
        return off;
      }
    }
    return -1;
  }
  void release(int64_t off, int64_t n) {
    if (n <= 0) return;
    used_ -= n;
    auto it = free_.emplace(off, n).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_.erase(nx);
    }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_.erase(it);
      }
    }
  }
  int64_t used() const { return used_; }

 private:
  std::map<int64_t, int64_t> free_;
  int64_t used_ = 0;
};

struct Job {
  int64_t id = 0;
  const bmadgpu_lattice* lat = nullptr;
  bmadgpu_bunch host;
  int32_t turn0 = 0, n_turns = 0;
  int32_t done_turns = 0;   // turns handed to rounds so far
  int32_t per_round = 1;    // turns per round
  int32_t slot = -1;
  int64_t off = -1;
  int32_t status = BMADGPU_JOB_QUEUED;
  int32_t rounds = 0;
  int64_t last_round = -1;  // last round the job has work in
  int64_t live = 0;         // live count after the last completed round
  bool retiring = false;
  double t_submit = -1, t_admit = -1, t_done = -1;
  int64_t particle_turns = 0;
  cudaEvent_t ev_up = nullptr, ev_down = nullptr;
  // frequency-map job: record range [rec_off, rec_off + rec_len) of the record arena (doubles),
  // parameters, result staging (pinned: tunes [6n] then rec_state [2n]) and the caller's points
  bool fma = false;
  int64_t rec_off = -1, rec_len = 0;
  int32_t fft_turns = 0, flip_a = 0, flip_b = 0;
  double rec_par[kRecPar] = {};
  void* h_fma = nullptr;
  bmadgpu_fma_point* fma_out = nullptr;
  double work() const { return (double)host.n * (double)(n_turns - done_turns) * (double)lat->pk.info.n_ele; }
};

struct Round {
  int64_t index;
  cudaEvent_t done;
  cudaEvent_t t0 = nullptr, t1 = nullptr;  // timing: the round's first and last operation
  int parity;                  // live list the round read
  std::vector<int64_t> jobs;   // jobs with work in the round
};

}  // namespace

struct bmadgpu_server {
  bmadgpu_ctx* ctx = nullptr;
  bmadgpu_server_config cfg;
  int64_t capacity = 0;
  cudaStream_t s_comp = nullptr, s_copy = nullptr;
  // device arena
  double* d_vec = nullptr;
  double* d_beta = nullptr;
  double* d_t = nullptr;
  int32_t* d_i32 = nullptr;  // state, ix_ele, ix_turn, location [4 * capacity]
  int32_t* d_live[2] = {nullptr, nullptr};
  BatchVar* d_vars = nullptr;
  unsigned long long* d_cnt = nullptr;  // [2][max_jobs]
  int64_t* d_prefix = nullptr;
  unsigned long long* d_queue = nullptr;
  // pinned mirrors, one per round in flight
  BatchVar* h_vars[kRoundsInFlight] = {nullptr, nullptr};
  unsigned long long* h_cnt[kRoundsInFlight] = {nullptr, nullptr};
  BatchKernel kern;
  uint32_t smem = 0;
  // record arena for frequency-map jobs (doubles)
  double* d_rec = nullptr;
  int64_t rec_capacity = 0;
  RangeAlloc rec_arena;
  // bookkeeping (guarded by mu)
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::unordered_map<int64_t, Job> jobs;
  std::deque<int64_t> queued;
  std::vector<int64_t> slot_job;  // job id per slot, -1 free
  RangeAlloc arena;
  int64_t next_id = 1;
  int64_t rounds = 0;
  int64_t submitted = 0, finished = 0, cancelled = 0;
  int64_t total_pt = 0;
  int64_t peak_resident = 0;
  double t_first = -1, t_last = -1;
  std::vector<double> latencies;
  // the compute stream's timeline: busy time of the rounds, the gaps between consecutive rounds
  cudaEvent_t t_ref = nullptr;
  double prev_end_ms = -1, busy_ms = 0, idle_ms = 0, max_gap_ms = 0;
  bool stop = false;
  int err_code = 0;
  std::string err_msg;
  std::thread worker;
};

namespace {

void set_error(bmadgpu_server* s, int code, const std::string& msg) {
  std::lock_guard<std::mutex> lk(s->mu);
  if (!s->err_code) {
    s->err_code = code;
    s->err_msg = msg;
  }
  s->cv_done.notify_all();
}

#define SRV_TRY(call)                                              \
  do {                                                             \
    cudaError_t e_ = (call);                                       \
    if (e_ != cudaSuccess) {                                       \
      set_error(s, BMADGPU_ECUDA, std::string(#call ": ") + cudaGetErrorString(e_)); \
      return false;                                                \
    }                                                              \
  } while (0)

BatchVar make_var(const Job& j) {
  BatchVar v;
  std::memset(&v, 0, sizeof(v));
  const bmadgpu_lattice* L = j.lat;
  v.table = L->d_table;
  v.ref_prefix = L->d_prefix;
  v.n = j.host.n;
  v.off = j.off;
  v.table_bytes = L->pk.info.total_bytes;
  v.hdr_bytes = L->pk.info.hdr_bytes;
  v.ap_bytes = L->pk.info.ap_bytes;
  v.n_ele = L->pk.info.n_ele;
  v.G = L->G;
  return v;
}

// The record pointers of a frequency-map job's descriptor.
void set_rec(BatchVar& v, const Job& j, double* d_rec) {
  const int64_t n = j.host.n, T = j.n_turns;
  double* base = d_rec + j.rec_off;
  v.rec = base;
  v.rec_par = base + 6 * T * n;
  v.rec_state = reinterpret_cast<int32_t*>(base + 6 * T * n + kRecPar + 6 * n);
  v.rec_turn0 = j.turn0;
  v.rec_turns = j.n_turns;
}

// Copies a job's particles into its arena range (copy stream) and records ev_up.
bool upload(bmadgpu_server* s, Job& j) {
  const int64_t n = j.host.n, off = j.off, C = s->capacity;
  const size_t nd = (size_t)n * sizeof(double), ni = (size_t)n * sizeof(int32_t);
  cudaStream_t st = s->s_copy;
  // vec of a job is its own [6][n] block at vec + 6 * off
  SRV_TRY(cudaMemcpyAsync(s->d_vec + 6 * off, j.host.vec, 6 * nd, cudaMemcpyHostToDevice, st));
  SRV_TRY(cudaMemcpyAsync(s->d_beta + off, j.host.beta, nd, cudaMemcpyHostToDevice, st));
  if (j.host.t) SRV_TRY(cudaMemcpyAsync(s->d_t + off, j.host.t, nd, cudaMemcpyHostToDevice, st));
  else SRV_TRY(cudaMemsetAsync(s->d_t + off, 0, nd, st));
  SRV_TRY(cudaMemcpyAsync(s->d_i32 + off, j.host.state, ni, cudaMemcpyHostToDevice, st));
  int32_t* ie = s->d_i32 + C + off;
  int32_t* it = s->d_i32 + 2 * C + off;
  int32_t* lo = s->d_i32 + 3 * C + off;
  if (j.host.ix_ele) SRV_TRY(cudaMemcpyAsync(ie, j.host.ix_ele, ni, cudaMemcpyHostToDevice, st));
  if (j.host.ix_turn) SRV_TRY(cudaMemcpyAsync(it, j.host.ix_turn, ni, cudaMemcpyHostToDevice, st));
  if (j.host.location) SRV_TRY(cudaMemcpyAsync(lo, j.host.location, ni, cudaMemcpyHostToDevice, st));
  if (j.fma) {
    BatchVar v;
    std::memset(&v, 0, sizeof(v));
    set_rec(v, j, s->d_rec);
    SRV_TRY(cudaMemcpyAsync(const_cast<double*>(v.rec_par), j.rec_par, sizeof(j.rec_par), cudaMemcpyHostToDevice, st));
    SRV_TRY(cudaMemsetAsync(v.rec_state, 0, 2 * ni, st));
  }
  SRV_TRY(cudaEventRecord(j.ev_up, st));
  return true;
}

bool download(bmadgpu_server* s, Job& j, cudaEvent_t after) {
  const int64_t n = j.host.n, off = j.off, C = s->capacity;
  const size_t nd = (size_t)n * sizeof(double), ni = (size_t)n * sizeof(int32_t);
  cudaStream_t st = s->s_copy;
  SRV_TRY(cudaStreamWaitEvent(st, after, 0));
  SRV_TRY(cudaMemcpyAsync(j.host.vec, s->d_vec + 6 * off, 6 * nd, cudaMemcpyDeviceToHost, st));
  SRV_TRY(cudaMemcpyAsync(j.host.beta, s->d_beta + off, nd, cudaMemcpyDeviceToHost, st));
  if (j.host.t) SRV_TRY(cudaMemcpyAsync(j.host.t, s->d_t + off, nd, cudaMemcpyDeviceToHost, st));
  SRV_TRY(cudaMemcpyAsync(j.host.state, s->d_i32 + off, ni, cudaMemcpyDeviceToHost, st));
  if (j.host.ix_ele) SRV_TRY(cudaMemcpyAsync(j.host.ix_ele, s->d_i32 + C + off, ni, cudaMemcpyDeviceToHost, st));
  if (j.host.ix_turn) SRV_TRY(cudaMemcpyAsync(j.host.ix_turn, s->d_i32 + 2 * C + off, ni, cudaMemcpyDeviceToHost, st));
  if (j.host.location)
    SRV_TRY(cudaMemcpyAsync(j.host.location, s->d_i32 + 3 * C + off, ni, cudaMemcpyDeviceToHost, st));
  if (j.fma) {
    // the tunes of the job's record, on the copy stream after the job's last round
    BatchVar v;
    std::memset(&v, 0, sizeof(v));
    set_rec(v, j, s->d_rec);
    double* tunes = v.rec + 6 * (int64_t)j.n_turns * n + kRecPar;
    int32_t* fstate = v.rec_state + 2 * n;
    SRV_TRY(fma_launch_tunes(v.rec, n, j.n_turns, j.fft_turns, s->d_i32 + off, v.rec_state, fstate, j.flip_a,
                             j.flip_b, tunes, s->ctx->sm_count, st));
    SRV_TRY(cudaMemcpyAsync(j.h_fma, tunes, 6 * nd, cudaMemcpyDeviceToHost, st));
    SRV_TRY(cudaMemcpyAsync((double*)j.h_fma + 6 * n, v.rec_state, 2 * ni, cudaMemcpyDeviceToHost, st));
  }
  SRV_TRY(cudaEventRecord(j.ev_down, st));
  return true;
}

// The caller's frequency-map points from the downloaded bunch and the staged tunes.
void fill_fma(const Job& j) {
  const int64_t n = j.host.n;
  const double* tunes = (const double*)j.h_fma;
  const int32_t* rs = (const int32_t*)(tunes + 6 * n);
  for (int64_t i = 0; i < n; ++i) {
    bmadgpu_fma_point& o = j.fma_out[i];
    std::memset(&o, 0, sizeof(o));
    if (rs[i] != 0) {  // stopped outside the bucket first (recording only runs while alive)
      o.status = rs[i];
      o.turn_lost = rs[n + i];
      o.ix_ele = -1;
    } else if (j.host.state[i] != 1) {
      o.status = 1;
      o.turn_lost = j.host.ix_turn ? j.host.ix_turn[i] - j.turn0 + 1 : -1;
      o.ix_ele = j.host.ix_ele ? j.host.ix_ele[i] : -1;
    } else {
      for (int k = 0; k < 6; ++k) o.tune[k] = tunes[i * 6 + k];
    }
  }
}

int64_t count_particle_turns(const Job& j) {
  // alive particles ran every turn; lost ones up to and including their loss turn
  int64_t pt = 0;
  for (int64_t i = 0; i < j.host.n; ++i) {
    if (j.host.state[i] == 1) pt += j.done_turns;
    else if (j.host.ix_turn && j.host.ix_turn[i] >= j.turn0) pt += j.host.ix_turn[i] - j.turn0 + 1;
  }
  return pt;
}

void worker_main(bmadgpu_server* s) {
  cudaSetDevice(s->ctx->device);
  std::deque<Round> inflight;
  int parity = 0;              // live list the next round reads
  std::vector<Job*> retiring;  // downloads enqueued, completion pending
  auto fail_all = [&]() {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
    s->cv_done.notify_all();
  };
  for (;;) {
    // ---- admission and round building (under the lock; CUDA calls only enqueue) ----------
    std::unique_lock<std::mutex> lk(s->mu);
    int64_t resident_live = 0;
    for (int64_t id : s->slot_job)
      if (id >= 0) resident_live += s->jobs[id].live;
    std::vector<int64_t> order(s->queued.begin(), s->queued.end());
    if (s->cfg.policy == BMADGPU_SERVE_SRPT)
      std::stable_sort(order.begin(), order.end(),
                       [&](int64_t a, int64_t b) { return s->jobs[a].work() < s->jobs[b].work(); });
    std::vector<int64_t> admitted;
    std::vector<Job*> admitted_jobs;  // element references stay valid: jobs are never erased
    for (int64_t id : order) {
      Job& j = s->jobs[id];
      if (resident_live > 0 && resident_live + j.host.n > s->cfg.target_live) break;
      auto free_slot = std::find(s->slot_job.begin(), s->slot_job.end(), (int64_t)-1);
      if (free_slot == s->slot_job.end()) break;
      const int64_t off = s->arena.alloc(j.host.n);
      if (off < 0) {
        if (s->cfg.policy == BMADGPU_SERVE_FIFO) break;
        continue;  // a smaller job may still fit
      }
      if (j.fma) {
        const int64_t roff = s->rec_arena.alloc(j.rec_len);
        if (roff < 0) {
          s->arena.release(off, j.host.n);
          if (s->cfg.policy == BMADGPU_SERVE_FIFO) break;
          continue;
        }
        j.rec_off = roff;
      }
      j.slot = (int32_t)(free_slot - s->slot_job.begin());
      j.off = off;
      *free_slot = id;
      j.status = BMADGPU_JOB_RUNNING;
      j.t_admit = now_s();
      j.live = j.host.n;
      resident_live += j.host.n;
      admitted.push_back(id);
      admitted_jobs.push_back(&j);
    }
    for (int64_t id : admitted) s->queued.erase(std::find(s->queued.begin(), s->queued.end(), id));
    s->peak_resident = std::max(s->peak_resident, s->arena.used());
    // jobs with turns left form the next round
    const int64_t r = s->rounds;
    const int buf = (int)(r % kRoundsInFlight);
    int32_t n_var = 0;
    std::vector<int64_t> round_jobs;
    bool round_records = false;
    int32_t round_rare = 0;
    for (int32_t slot = 0; slot < (int32_t)s->slot_job.size(); ++slot) {
      const int64_t id = s->slot_job[slot];
      BatchVar& hv = s->h_vars[buf][slot];
      std::memset(&hv, 0, sizeof(hv));
      if (id < 0) continue;
      Job& j = s->jobs[id];
      n_var = slot + 1;
      hv = make_var(j);
      if (j.lat->pk.info.rare) round_rare = 1;
      if (j.fma) set_rec(hv, j, s->d_rec);
      const int32_t left = j.n_turns - j.done_turns;
      if (left <= 0 || j.retiring || j.live == 0) continue;
      const int32_t k = std::min(left, j.per_round);
      hv.turn0 = j.turn0 + j.done_turns;
      hv.n_turns = k;
      j.done_turns += k;
      j.rounds++;
      j.last_round = r;
      round_jobs.push_back(id);
      round_records = round_records || j.fma;
    }
    const bool stopping = s->stop;
    lk.unlock();
    (void)stopping;

    // ---- enqueue: uploads (copy stream), first live lists, the round (compute stream) --------
    bool ok = true;
    for (Job* jp : admitted_jobs) {
      Job& j = *jp;  // only the worker mutates running jobs
      ok = ok && upload(s, j);
      if (ok && cudaStreamWaitEvent(s->s_comp, j.ev_up, 0) != cudaSuccess) ok = false;
      if (ok && batch_launch_init_list(s->d_live[parity] + j.off, j.host.n,
                                       s->d_cnt + (size_t)parity * s->cfg.max_jobs + j.slot, s->s_comp) != cudaSuccess)
        ok = false;
    }
    if (!ok) {
      set_error(s, BMADGPU_ECUDA, "server: admission failed");
      fail_all();
      return;
    }
    if (!round_jobs.empty()) {
      const size_t J = (size_t)s->cfg.max_jobs;
      cudaStream_t c = s->s_comp;
      BatchArgs a;
      std::memset(&a, 0, sizeof(a));
      a.vars = s->d_vars;
      a.n_var = n_var;
      a.tile = s->kern.block * s->kern.ppt;
      a.vec = s->d_vec;
      a.beta = s->d_beta;
      a.t = s->d_t;
      a.state = s->d_i32;
      a.ix_ele = s->d_i32 + s->capacity;
      a.ix_turn = s->d_i32 + 2 * s->capacity;
      a.location = s->d_i32 + 3 * s->capacity;
      a.turn_off = 0;
      a.n_turns = 1 << 30;  // each job's own turns (BatchVar::n_turns) bound the round
      a.tile_prefix = s->d_prefix;
      a.live_in = s->d_live[parity];
      a.n_in = s->d_cnt + (size_t)parity * J;
      a.live_out = s->d_live[1 - parity];
      a.n_out = s->d_cnt + (size_t)(1 - parity) * J;
      a.queue = s->d_queue;
      a.err_flag = s->ctx->d_err;
      a.smem_bytes = s->smem;
      a.rare = round_rare;
      Round rd;
      rd.index = r;
      rd.parity = parity;
      rd.jobs = round_jobs;
      rd.done = nullptr;
      ok = cudaEventCreate(&rd.t0) == cudaSuccess && cudaEventCreate(&rd.t1) == cudaSuccess &&
           cudaEventRecord(rd.t0, c) == cudaSuccess &&
           cudaMemcpyAsync(s->d_vars, s->h_vars[buf], sizeof(BatchVar) * n_var, cudaMemcpyHostToDevice, c) ==
               cudaSuccess &&
           batch_launch_plan(s->d_vars, n_var, a.tile, 0, false, a.n_in, s->d_prefix, s->d_queue, a.n_out, c) ==
               cudaSuccess &&
           batch_launch_track(s->kern, a, c, round_records) == cudaSuccess &&
           cudaMemcpyAsync(s->h_cnt[buf], a.n_out, sizeof(unsigned long long) * n_var, cudaMemcpyDeviceToHost, c) ==
               cudaSuccess &&
           cudaEventRecord(rd.t1, c) == cudaSuccess &&
           cudaEventCreateWithFlags(&rd.done, cudaEventDisableTiming) == cudaSuccess &&
           cudaEventRecord(rd.done, c) == cudaSuccess;
      if (!ok) {
        set_error(s, BMADGPU_ECUDA, "server: round launch failed");
        fail_all();
        return;
      }
      inflight.push_back(rd);
      parity = 1 - parity;
      lk.lock();
      s->rounds++;
      lk.unlock();
    }

    // ---- complete the oldest round when the pipeline is full (or nothing else can be queued) --
    const bool must_wait = (int)inflight.size() >= kRoundsInFlight || (round_jobs.empty() && !inflight.empty());
    if (must_wait) {
      Round rd = inflight.front();
      inflight.pop_front();
      if (cudaEventSynchronize(rd.done) != cudaSuccess) {
        set_error(s, BMADGPU_ECUDA, "server: round failed");
        fail_all();
        return;
      }
      const int b = (int)(rd.index % kRoundsInFlight);
      {
        // rounds run one after another on the compute stream: their busy time, and the gaps in
        // which the stream waited for the worker (admission, bookkeeping) or for work
        if (!s->t_ref) {
          s->t_ref = rd.t0;
          rd.t0 = nullptr;
        }
        float a_ms = 0, b_ms = 0;
        if (rd.t0) cudaEventElapsedTime(&a_ms, s->t_ref, rd.t0);
        cudaEventElapsedTime(&b_ms, s->t_ref, rd.t1);
        lk.lock();
        s->busy_ms += b_ms - a_ms;
        if (s->prev_end_ms >= 0 && a_ms > s->prev_end_ms) {
          s->idle_ms += a_ms - s->prev_end_ms;
          s->max_gap_ms = std::max(s->max_gap_ms, (double)(a_ms - s->prev_end_ms));
        }
        s->prev_end_ms = b_ms;
        lk.unlock();
        if (rd.t0) cudaEventDestroy(rd.t0);
        cudaEventDestroy(rd.t1);
      }
      std::vector<Job*> finishing;
      lk.lock();
      for (int64_t id : rd.jobs) {
        Job& j = s->jobs[id];
        if (j.retiring) continue;
        j.live = (int64_t)s->h_cnt[b][j.slot];
        // Done when this was its last round, or when nothing is left alive (it may then still be
        // listed in the next in-flight round, but with a zero live count, so no kernel touches it).
        if ((j.done_turns >= j.n_turns && j.last_round == rd.index) || j.live == 0) {
          j.retiring = true;
          finishing.push_back(&j);
        }
      }
      lk.unlock();
      for (Job* jp : finishing) {
        Job& j = *jp;
        if (!download(s, j, rd.done)) {
          fail_all();
          return;
        }
        lk.lock();
        // Slot and range are free for waiting jobs now: their uploads follow this download on the
        // copy stream, and no round in flight has work for this job.
        s->slot_job[j.slot] = -1;
        s->arena.release(j.off, j.host.n);
        if (j.fma) s->rec_arena.release(j.rec_off, j.rec_len);
        lk.unlock();
        retiring.push_back(jp);
      }
      cudaEventDestroy(rd.done);
    }

    // ---- completions: result copies that have landed -----------------------------------------
    std::vector<Job*> still;
    for (Job* jp : retiring) {
      Job& j = *jp;
      cudaError_t q = cudaEventQuery(j.ev_down);
      if (q == cudaErrorNotReady) {
        still.push_back(jp);
        continue;
      }
      if (q != cudaSuccess) {
        set_error(s, BMADGPU_ECUDA, "server: result copy failed");
        fail_all();
        return;
      }
      const int64_t pt = count_particle_turns(j);
      if (j.fma) fill_fma(j);
      lk.lock();
      j.particle_turns = pt;
      j.t_done = now_s();
      j.status = BMADGPU_JOB_DONE;
      s->finished++;
      s->total_pt += pt;
      s->t_last = j.t_done;
      s->latencies.push_back(j.t_done - j.t_submit);
      s->cv_done.notify_all();
      lk.unlock();
    }
    retiring.swap(still);

    // ---- idle: nothing resident, nothing queued ------------------------------------------------
    lk.lock();
    bool resident = false;
    for (int64_t id : s->slot_job) resident = resident || id >= 0;
    const bool idle = !resident && inflight.empty() && retiring.empty();
    if (idle && s->queued.empty()) {
      if (stopping || s->stop) {
        lk.unlock();
        return;
      }
      s->cv_work.wait_for(lk, std::chrono::milliseconds(20));
    } else if (round_jobs.empty() && admitted.empty() && !must_wait) {
      // only result copies pending, or queued jobs waiting for space: poll gently
      s->cv_work.wait_for(lk, std::chrono::microseconds(200));
    }
    lk.unlock();
  }
}

}  // namespace

extern "C" {

int bmadgpu_host_alloc(int64_t bytes, void** ptr) {
  if (!ptr || bytes < 0) return fail(BMADGPU_EINVAL, "bad argument");
  *ptr = nullptr;
  if (bytes == 0) return BMADGPU_OK;
  if (cudaHostAlloc(ptr, (size_t)bytes, cudaHostAllocPortable) != cudaSuccess) {
    *ptr = nullptr;
    return fail(BMADGPU_ENOMEM, "cudaHostAlloc failed");
  }
  return BMADGPU_OK;
}

int bmadgpu_host_free(void* ptr) {
  if (ptr) CUDA_TRY(cudaFreeHost(ptr));
  return BMADGPU_OK;
}

int bmadgpu_server_create(bmadgpu_ctx* c, const bmadgpu_server_config* cfg_in, bmadgpu_server** out) {
  if (!c || !out) return fail(BMADGPU_EINVAL, "NULL argument");
  *out = nullptr;
  bmadgpu_server_config cfg;
  std::memset(&cfg, 0, sizeof(cfg));
  if (cfg_in) cfg = *cfg_in;
  if (cfg.max_particles < 0 || cfg.hbm_fraction < 0 || cfg.hbm_fraction > 0.95 || cfg.max_jobs < 0 ||
      cfg.element_steps < 0 || cfg.target_live < 0 || (cfg.policy != BMADGPU_SERVE_SRPT && cfg.policy != BMADGPU_SERVE_FIFO))
    return fail(BMADGPU_EINVAL, "bad server configuration");
  if (cfg.hbm_fraction == 0) cfg.hbm_fraction = 0.5;
  if (cfg.max_jobs == 0) cfg.max_jobs = 4096;
  if (cfg.element_steps == 0) cfg.element_steps = 4096;
  if (cfg.target_live == 0) cfg.target_live = 1 << 20;
  if (cfg.block == 0) {
    // 128 x 4 measured fastest on the mixed request stream (200 jobs: 1.59e7 particle-turns/s
    // against 1.45e7 for 64 x 12 and 1.57e7 for 256 x 2)
    cfg.block = 128;
    if (cfg.ctas_per_sm == 0) cfg.ctas_per_sm = 4;
  }
  CUDA_TRY(cudaSetDevice(c->device));
  size_t free_b = 0, total_b = 0;
  CUDA_TRY(cudaMemGetInfo(&free_b, &total_b));
  int64_t cap = cfg.max_particles;
  const int64_t by_hbm = (int64_t)((double)free_b * cfg.hbm_fraction / (double)kBytesPerParticle);
  if (cap == 0 || cap > by_hbm) cap = by_hbm;
  if (cap > 0x7fffffffLL) cap = 0x7fffffffLL;
  if (cap < 1) return fail(BMADGPU_ENOMEM, "no device memory for the particle arena");
  bmadgpu_server* s = new (std::nothrow) bmadgpu_server();
  if (!s) return fail(BMADGPU_ENOMEM, "host allocation failed");
  s->ctx = c;
  s->cfg = cfg;
  s->capacity = cap;
  s->arena.reset(cap);
  s->slot_job.assign(cfg.max_jobs, -1);
  const size_t C = (size_t)cap, J = (size_t)cfg.max_jobs;
  bool ok = cudaStreamCreateWithFlags(&s->s_comp, cudaStreamNonBlocking) == cudaSuccess &&
            cudaStreamCreateWithFlags(&s->s_copy, cudaStreamNonBlocking) == cudaSuccess &&
            cudaMalloc(&s->d_vec, 6 * C * sizeof(double)) == cudaSuccess &&
            cudaMalloc(&s->d_beta, C * sizeof(double)) == cudaSuccess &&
            cudaMalloc(&s->d_t, C * sizeof(double)) == cudaSuccess &&
            cudaMalloc(&s->d_i32, 4 * C * sizeof(int32_t)) == cudaSuccess &&
            cudaMalloc(&s->d_live[0], C * sizeof(int32_t)) == cudaSuccess &&
            cudaMalloc(&s->d_live[1], C * sizeof(int32_t)) == cudaSuccess &&
            cudaMalloc(&s->d_vars, J * sizeof(BatchVar)) == cudaSuccess &&
            cudaMalloc(&s->d_cnt, 2 * J * sizeof(unsigned long long)) == cudaSuccess &&
            cudaMalloc(&s->d_prefix, (J + 1) * sizeof(int64_t)) == cudaSuccess &&
            cudaMalloc(&s->d_queue, sizeof(unsigned long long)) == cudaSuccess;
  for (int i = 0; ok && i < kRoundsInFlight; ++i)
    ok = cudaHostAlloc(&s->h_vars[i], J * sizeof(BatchVar), cudaHostAllocPortable) == cudaSuccess &&
         cudaHostAlloc(&s->h_cnt[i], J * sizeof(unsigned long long), cudaHostAllocPortable) == cudaSuccess;
  ok = ok && cudaMemset(s->d_cnt, 0, 2 * J * sizeof(unsigned long long)) == cudaSuccess;
  if (ok) {
    // record arena for frequency-map jobs: record_mib, or a quarter of what is free now
    size_t free2 = 0, total2 = 0;
    ok = cudaMemGetInfo(&free2, &total2) == cudaSuccess;
    const double want = cfg.record_mib > 0 ? (double)cfg.record_mib * 1048576.0 : 0.25 * (double)free2;
    const int64_t cap_rec = (int64_t)(std::min(want, 0.9 * (double)free2) / sizeof(double));
    if (ok && cap_rec > 0 && cudaMalloc(&s->d_rec, (size_t)cap_rec * sizeof(double)) == cudaSuccess) {
      s->rec_capacity = cap_rec;
      s->rec_arena.reset(cap_rec);
    } else {
      cudaGetLastError();
      s->rec_arena.reset(0);
    }
  }
  if (ok) {
    s->smem = cfg.stage_smem ? kServeStageBytes : 0;
    BatchLaunch bl;
    bl.block = cfg.block;
    bl.ctas_per_sm = cfg.ctas_per_sm;
    bl.particles_per_thread = 1;
    ok = batch_resolve(bl, s->smem, c->sm_count, &s->kern) == cudaSuccess;
  }
  if (!ok) {
    bmadgpu_server_destroy(s);
    return fail(BMADGPU_ENOMEM, "cannot allocate the server's device state");
  }
  s->worker = std::thread(worker_main, s);
  *out = s;
  return BMADGPU_OK;
}

int bmadgpu_server_destroy(bmadgpu_server* s) {
  if (!s) return BMADGPU_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    for (int64_t id : s->queued) {
      s->jobs[id].status = BMADGPU_JOB_CANCELLED;
      s->cancelled++;
    }
    s->queued.clear();
    s->stop = true;
    s->cv_work.notify_all();
    s->cv_done.notify_all();
  }
  if (s->worker.joinable()) s->worker.join();
  cudaSetDevice(s->ctx->device);
  if (s->s_comp) cudaStreamSynchronize(s->s_comp);
  if (s->s_copy) cudaStreamSynchronize(s->s_copy);
  for (auto& kv : s->jobs) {
    if (kv.second.ev_up) cudaEventDestroy(kv.second.ev_up);
    if (s->t_ref) {
      cudaEventDestroy(s->t_ref);
      s->t_ref = nullptr;
    }
    if (kv.second.ev_down) cudaEventDestroy(kv.second.ev_down);
    if (kv.second.h_fma) cudaFreeHost(kv.second.h_fma);
  }
  cudaFree(s->d_rec);
  cudaFree(s->d_vec);
  cudaFree(s->d_beta);
  cudaFree(s->d_t);
  cudaFree(s->d_i32);
  cudaFree(s->d_live[0]);
  cudaFree(s->d_live[1]);
  cudaFree(s->d_vars);
  cudaFree(s->d_cnt);
  cudaFree(s->d_prefix);
  cudaFree(s->d_queue);
  for (int i = 0; i < kRoundsInFlight; ++i) {
    cudaFreeHost(s->h_vars[i]);
    cudaFreeHost(s->h_cnt[i]);
  }
  if (s->s_comp) cudaStreamDestroy(s->s_comp);
  if (s->s_copy) cudaStreamDestroy(s->s_copy);
  delete s;
  return BMADGPU_OK;
}

}  // extern "C"

namespace {

// Queues a job (fma: a frequency-map job with its prepared fields; nullptr otherwise).
int submit_job(bmadgpu_server* s, const bmadgpu_lattice* lat, bmadgpu_bunch* b, int32_t turn0, int32_t n_turns,
               const Job* fma, int64_t* job_id) {
  if (!s || !lat || !b || !job_id) return fail(BMADGPU_EINVAL, "NULL argument");
  if (b->n < 0 || n_turns < 0) return fail(BMADGPU_EINVAL, "negative particle or turn count");
  if (b->n > 0 && (!b->vec || !b->beta || !b->state)) return fail(BMADGPU_EINVAL, "bunch vec/beta/state NULL");
  if (lat->device != s->ctx->device) return fail(BMADGPU_EINVAL, "lattice and server are on different devices");
  if (b->n > s->capacity) return fail(BMADGPU_ENOMEM, "the bunch is larger than the server's particle arena");
  if (fma && fma->rec_len > s->rec_capacity)
    return fail(BMADGPU_ENOMEM, "the frequency-map record is larger than the server's record arena");
  cudaEvent_t up = nullptr, down = nullptr;
  CUDA_TRY(cudaSetDevice(s->ctx->device));
  CUDA_TRY(cudaEventCreateWithFlags(&up, cudaEventDisableTiming));
  if (cudaEventCreateWithFlags(&down, cudaEventDisableTiming) != cudaSuccess) {
    cudaEventDestroy(up);
    return fail(BMADGPU_ECUDA, "cudaEventCreate failed");
  }
  void* h_fma = nullptr;
  if (fma && b->n > 0 &&
      cudaHostAlloc(&h_fma, (size_t)b->n * (6 * sizeof(double) + 2 * sizeof(int32_t)), cudaHostAllocPortable) !=
          cudaSuccess) {
    cudaEventDestroy(up);
    cudaEventDestroy(down);
    return fail(BMADGPU_ENOMEM, "cudaHostAlloc failed");
  }
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->err_code || s->stop || s->queued.size() >= kMaxQueued) {
    cudaEventDestroy(up);
    cudaEventDestroy(down);
    if (h_fma) cudaFreeHost(h_fma);
    if (s->err_code) return fail(s->err_code, s->err_msg);
    return fail(BMADGPU_EBUSY, "server queue is full or stopping");
  }
  Job j;
  if (fma) j = *fma;
  j.id = s->next_id++;
  j.lat = lat;
  j.host = *b;
  j.turn0 = turn0;
  j.n_turns = n_turns;
  j.per_round = std::max<int32_t>(1, s->cfg.element_steps / std::max<int32_t>(1, (int32_t)lat->pk.info.n_ele));
  j.t_submit = now_s();
  j.ev_up = up;
  j.ev_down = down;
  j.h_fma = h_fma;
  if (s->t_first < 0) s->t_first = j.t_submit;
  s->submitted++;
  if (b->n == 0 || n_turns == 0) {
    // nothing to track: done at once
    j.status = BMADGPU_JOB_DONE;
    j.t_admit = j.t_done = j.t_submit;
    s->finished++;
    s->latencies.push_back(0.0);
    s->t_last = j.t_done;
  } else {
    s->queued.push_back(j.id);
  }
  *job_id = j.id;
  s->jobs.emplace(j.id, j);
  s->cv_work.notify_all();
  s->cv_done.notify_all();
  return BMADGPU_OK;
}

}  // namespace

extern "C" {

int bmadgpu_server_submit(bmadgpu_server* s, const bmadgpu_lattice* lat, bmadgpu_bunch* b, int32_t turn0,
                          int32_t n_turns, int64_t* job_id) {
  return submit_job(s, lat, b, turn0, n_turns, nullptr, job_id);
}

int bmadgpu_server_submit_fma(bmadgpu_server* s, const bmadgpu_lattice* lat, bmadgpu_bunch* b, int32_t turn0,
                              int32_t n_turns, const bmadgpu_fma_params* P, bmadgpu_fma_point* points,
                              int64_t* job_id) {
  if (!s || !lat || !b || !P || (b->n > 0 && !points)) return fail(BMADGPU_EINVAL, "NULL argument");
  if (n_turns < 2) return fail(BMADGPU_EINVAL, "a frequency-map job needs at least 2 turns");
  Job f;
  f.fma = true;
  f.fft_turns = P->fft_turns > 0 ? P->fft_turns : n_turns / 2;
  if (f.fft_turns < 2 || f.fft_turns > n_turns || f.fft_turns > 4096)
    return fail(BMADGPU_EINVAL, "fft_turns must be in [2, min(n_turns, 4096)]");
  f.flip_a = P->tune_a < 0.5;
  f.flip_b = P->tune_b < 0.5;
  std::memcpy(f.rec_par, P->norm, sizeof(double) * 36);
  std::memcpy(f.rec_par + 36, P->orbit, sizeof(double) * 6);
  double z_limit = 0;
  if (P->z_cut) {  // frequency_map.f90:99-119
    double fr = P->rf_frequency;
    if (fr <= 0) {
      fr = 0;
      for (const auto& e : lat->eles)
        if (e.key == BMADGPU_RFCAVITY) fr = (fr == 0) ? e.rf_frequency : std::fmin(fr, e.rf_frequency);
    }
    if (fr > 0) z_limit = 0.25 * (299792458.0 / fr);
  }
  f.rec_par[42] = z_limit;
  f.rec_len = rec_doubles(b->n, n_turns);
  f.fma_out = points;
  return submit_job(s, lat, b, turn0, n_turns, &f, job_id);
}

int bmadgpu_server_job(bmadgpu_server* s, int64_t id, bmadgpu_job_info* info) {
  if (!s || !info) return fail(BMADGPU_EINVAL, "NULL argument");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->jobs.find(id);
  if (it == s->jobs.end()) return fail(BMADGPU_ENOTFOUND, "unknown job id");
  const Job& j = it->second;
  info->status = j.status;
  info->rounds = j.rounds;
  const double t0 = s->t_first;
  info->t_submit = j.t_submit - t0;
  info->t_admit = j.t_admit < 0 ? -1 : j.t_admit - t0;
  info->t_done = j.t_done < 0 ? -1 : j.t_done - t0;
  info->particle_turns = j.particle_turns;
  return BMADGPU_OK;
}

int bmadgpu_server_wait(bmadgpu_server* s, int64_t id, double timeout_s) {
  if (!s) return fail(BMADGPU_EINVAL, "server is NULL");
  std::unique_lock<std::mutex> lk(s->mu);
  if (id != -1 && s->jobs.find(id) == s->jobs.end()) return fail(BMADGPU_ENOTFOUND, "unknown job id");
  auto done = [&]() {
    if (s->err_code) return true;
    if (id == -1) return s->finished + s->cancelled >= s->submitted;
    const int st = s->jobs[id].status;
    return st == BMADGPU_JOB_DONE || st == BMADGPU_JOB_CANCELLED;
  };
  const auto deadline = std::chrono::steady_clock::now() + std::chrono::duration<double>(timeout_s);
  while (!done()) {
    if (s->cv_done.wait_until(lk, deadline) == std::cv_status::timeout && !done())
      return fail(BMADGPU_ETIMEDOUT, "server wait timed out");
  }
  if (s->err_code) return fail(s->err_code, s->err_msg);
  return BMADGPU_OK;
}

int bmadgpu_server_get_stats(bmadgpu_server* s, bmadgpu_server_stats* st) {
  if (!s || !st) return fail(BMADGPU_EINVAL, "NULL argument");
  std::lock_guard<std::mutex> lk(s->mu);
  std::memset(st, 0, sizeof(*st));
  st->jobs_submitted = s->submitted;
  st->jobs_done = s->finished;
  st->rounds = s->rounds;
  st->particle_turns = s->total_pt;
  st->elapsed_s = (s->t_first >= 0 && s->t_last >= 0) ? s->t_last - s->t_first : 0.0;
  st->capacity = s->capacity;
  st->peak_resident = s->peak_resident;
  st->gpu_busy_s = s->busy_ms / 1e3;
  st->gpu_idle_s = s->idle_ms / 1e3;
  st->gpu_max_gap_s = s->max_gap_ms / 1e3;
  if (!s->latencies.empty()) {
    std::vector<double> l = s->latencies;
    std::sort(l.begin(), l.end());
    auto q = [&](double p) {
      // nearest-rank percentile
      size_t k = (size_t)std::ceil(p * (double)l.size());
      if (k < 1) k = 1;
      return l[k - 1];
    };
    st->latency_p50_s = q(0.50);
    st->latency_p99_s = q(0.99);
    st->latency_max_s = l.back();
  }
  return BMADGPU_OK;
}

}  // extern "C"
