/*
 * bmadgpu.h -- C-ABI of the B200 (sm_100a, FP64) multi-particle tracker.
 *
 * This is the drop-in boundary for Bmad's multi-particle bmad_standard tracking path
 * (track_bunch -> track1_bunch -> track1_bunch_hom -> track1 -> track1_bmad -> track_a_*).
 * Every entry point is plain C: pointers, sizes and status codes, no C++ or torch types.
 *
 * Reference interfaces replaced (paths inside bmad-sim/bmad-ecosystem):
 *   - track1_bunch_hook_ptr / track1_bunch_hook          bmad/custom/track1_bunch_hook.f90:25-43,
 *                                                         called at bmad/multiparticle/beam_mod.f90:263-266
 *   - track_bunch (element loop over a branch)           bmad/multiparticle/beam_mod.f90:103-170
 *   - ltt_run_beam_mode turn loop + ltt_track_bmad_bunch bsim/modules/lt_tracking_mod.f90:1631-1713, 3189-3224
 *   - track1_bunch_hom OpenMP particle loop               bmad/multiparticle/beam_utils.f90:81-86
 *   - coord_struct / bunch_struct marshalling             bmad/modules/bmad_struct.f90:551-579, 1117-1135
 *     (component-wise, as cpp_bmad_interface/code/bmad_cpp_convert_mod.f90:1767-1844 does)
 *
 * Units and conventions are Bmad's: vec = (x, px, y, py, z, pz) canonical, px/py normalised by
 * p0c, pz = (p - p0)/p0, z = -beta*c*(t - t_ref). Integer enums below carry Bmad's own values so a
 * Fortran caller can pass ele%key, ele%value(fringe_type$), coord%state, ... unchanged.
 *
 * Status: every function returns 0 on success or a negative BMADGPU_E* code; the message of the
 * last failure on the calling host thread is available from bmadgpu_last_error().
 */
#ifndef BMADGPU_H
#define BMADGPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BMADGPU_ABI_VERSION 1
#define BMADGPU_N_POLE 22          /* multipole arrays 0:n_pole_maxx, n_pole_maxx = 21 (bmad_struct.f90:48) */
#define BMADGPU_N_MOMENTS 28       /* per reported turn: n_live, sum vec_i (6), sum vec_i vec_j i<=j (21) */

/* ---- status codes ------------------------------------------------------------------------ */
enum {
  BMADGPU_OK = 0,
  BMADGPU_EINVAL = -1,        /* bad argument (null pointer, n < 0, inconsistent sizes) */
  BMADGPU_ENOMEM = -2,        /* device or pinned-host allocation failed, or admission refused */
  BMADGPU_ECUDA = -3,         /* a CUDA runtime call failed */
  BMADGPU_ETIMEDOUT = -4,     /* a bounded device/host wait ran out */
  BMADGPU_EUNSUPPORTED = -5,  /* element type, flag or method outside the bmad_standard hot path */
  BMADGPU_EBUSY = -6,         /* serving queue full */
  BMADGPU_ENOTFOUND = -7      /* unknown job id */
};

/* ---- Bmad enum values (bmad/modules/bmad_struct.f90) ---------------------------------------- */
/* element keys, bmad_struct.f90:1696-1710 */
enum {
  BMADGPU_DRIFT = 1, BMADGPU_SBEND = 2, BMADGPU_QUADRUPOLE = 3, BMADGPU_SEXTUPOLE = 5,
  BMADGPU_RFCAVITY = 9, BMADGPU_MARKER = 14, BMADGPU_OCTUPOLE = 17, BMADGPU_MULTIPOLE = 19,
  BMADGPU_AB_MULTIPOLE = 22, BMADGPU_MONITOR = 31, BMADGPU_INSTRUMENT = 32, BMADGPU_PIPE = 44,
  BMADGPU_THICK_MULTIPOLE = 67, BMADGPU_RCOLLIMATOR = 35, BMADGPU_ECOLLIMATOR = 36,
  BMADGPU_KICKER = 15, BMADGPU_HKICKER = 33, BMADGPU_VKICKER = 34, BMADGPU_ELSEPARATOR = 10
};
/* particle states, bmad_struct.f90:525-532 */
enum {
  BMADGPU_ALIVE = 1, BMADGPU_LOST = 2, BMADGPU_LOST_NEG_X = 3, BMADGPU_LOST_POS_X = 4,
  BMADGPU_LOST_NEG_Y = 5, BMADGPU_LOST_POS_Y = 6, BMADGPU_LOST_Z = 7, BMADGPU_LOST_PZ = 8
};
/* coord%location, bmad_struct.f90:376-377 */
enum { BMADGPU_UPSTREAM_END = 1, BMADGPU_DOWNSTREAM_END = 2, BMADGPU_INSIDE = 3 };
/* fringe_at / aperture_at, bmad_struct.f90:373-374 */
enum {
  BMADGPU_ENTRANCE_END = 1, BMADGPU_EXIT_END = 2, BMADGPU_BOTH_ENDS = 3, BMADGPU_NO_END = 4,
  BMADGPU_CONTINUOUS = 5
};
/* fringe_type, bmad_struct.f90:27, 168-169 */
enum {
  BMADGPU_FRINGE_NONE = 1, BMADGPU_FRINGE_SOFT_EDGE_ONLY = 2, BMADGPU_FRINGE_HARD_EDGE_ONLY = 3,
  BMADGPU_FRINGE_FULL = 4, BMADGPU_FRINGE_SAD_FULL = 5, BMADGPU_FRINGE_LINEAR_EDGE = 6,
  BMADGPU_FRINGE_BASIC_BEND = 7
};
/* aperture_type, bmad_struct.f90:158 */
enum { BMADGPU_APERTURE_AUTO = 1, BMADGPU_APERTURE_RECTANGULAR = 2, BMADGPU_APERTURE_ELLIPTICAL = 3 };

/* ---- lattice element -------------------------------------------------------------------------
 * One record per tracked element, in tracking order (branch%ele(1:n_ele_track)). Field names are
 * the ele%value(...) attribute names. Defaults a caller must set explicitly (there is no parser):
 * sbend fringe_type = basic_bend, every other element none; fringe_at = both_ends;
 * aperture_at = exit_end; aperture_type = rectangular; scale_multipoles = 1; is_on = 1;
 * fintx/hgapx = fint/hgap when unset (set_ele_defaults.f90:36-37, 295-300;
 * bmad_parser_mod.f90:5238-5239).
 * For key = multipole, a_pole holds knl(0:21) and b_pole holds tn(0:21) as in Bmad.
 */
typedef struct bmadgpu_element {
  int32_t key;
  int32_t is_on;
  int32_t fringe_type;
  int32_t fringe_at;
  int32_t aperture_at;
  int32_t aperture_type;
  int32_t num_steps;          /* 0 => computed as attribute_bookkeeper.f90:292-400 does */
  int32_t scale_multipoles;
  int32_t field_master;       /* must be 0 (normalised strengths) */
  int32_t exact_multipoles;   /* must be off$ (= 1) or 0 */
  int32_t orientation;        /* must be +1 */
  int32_t reserved;
  double l, k1, k2, k3, g, dg, e1, e2, fint, fintx, hgap, hgapx;
  double tilt, ref_tilt, roll, x_offset, y_offset, z_offset, x_pitch, y_pitch;
  double hkick, vkick;
  double x1_limit, x2_limit, y1_limit, y2_limit;
  double voltage, rf_frequency, phi0, phi0_multipass;
  double ds_step, r0_mag, r0_elec;
  double delta_ref_time;      /* ele%value(delta_ref_time$); used only for the time coordinate */
  double a_pole[BMADGPU_N_POLE], b_pole[BMADGPU_N_POLE];
  double a_pole_elec[BMADGPU_N_POLE], b_pole_elec[BMADGPU_N_POLE];
  double fq1, fq2;            /* quadrupole soft-edge fringe integrals (soft_quadrupole_edge_kick) */
  /* collimator phase-space windows (check_aperture_limit.f90:115-151): half widths and centres in
   * px, py, z, pz; a zero half width leaves that coordinate unchecked */
  double px_aperture_width2, px_aperture_center, py_aperture_width2, py_aperture_center;
  double z_aperture_width2, z_aperture_center, pz_aperture_width2, pz_aperture_center;
  double kick;                /* hkicker / vkicker: ele%value(kick$) */
} bmadgpu_element;

/* Branch/global parameters: lat_param_struct + the bmad_common_struct switches on the path. */
typedef struct bmadgpu_param {
  double p0c;                 /* reference momentum [eV], ele%value(p0c$) (constant along the ring) */
  double e_tot;               /* reference total energy [eV], ele%value(e_tot$) */
  double mass;                /* mass_of(species) [eV] */
  double charge;              /* charge_of(species) [e] */
  double max_aperture_limit;  /* bmad_com%max_aperture_limit, default 1e3 */
  double default_ds_step;     /* bmad_com%default_ds_step, default 0.2 */
  int32_t aperture_limit_on;  /* bmad_com%aperture_limit_on, default 1 */
  int32_t absolute_time_tracking; /* must be 0 (relative time, bmad_struct.f90:2350) */
  int32_t radiation_on;       /* must be 0: radiation, spin, wakes, space charge are off the path */
  int32_t reserved;
} bmadgpu_param;

/* Particles in structure-of-arrays form; the Fortran shim gathers coord_struct fields into it. */
typedef struct bmadgpu_bunch {
  int64_t n;                  /* number of particles */
  double* vec;                /* [6*n]: vec[i*n + j] = coordinate i (0..5) of particle j */
  double* beta;               /* [n]: coord%beta */
  double* t;                  /* [n] or NULL: coord%t (FP64; the reference keeps it in real(qp)) */
  int32_t* state;             /* [n]: coord%state */
  int32_t* ix_ele;            /* [n] or NULL: element index (0-based) of the loss; untouched if alive */
  int32_t* ix_turn;           /* [n] or NULL: turn index of the loss; untouched if alive */
  int32_t* location;          /* [n] or NULL: coord%location at the loss */
} bmadgpu_bunch;

typedef struct bmadgpu_ctx bmadgpu_ctx;
typedef struct bmadgpu_lattice bmadgpu_lattice;

/* ---- library, context, lattice -------------------------------------------------------------- */
int bmadgpu_abi_version(void);
const char* bmadgpu_last_error(void);

/* One context per host thread and device; it owns a CUDA stream and device scratch. */
int bmadgpu_ctx_create(int32_t device, bmadgpu_ctx** out);
/* Destroy a context only after the batches and servers made on it (their destroy calls use the
 * context's stream); lattices may outlive it. */
int bmadgpu_ctx_destroy(bmadgpu_ctx* ctx);

/* Packs the element records into the device element table (per-element invariants hoisted,
 * n_step bookkeeping as attribute_bookkeeper.f90:292-400, multipoles as
 * multipole_ele_to_ab.f90:31-678). Replaces what branch%ele(:) provides to track1. */
int bmadgpu_lattice_create(bmadgpu_ctx* ctx, const bmadgpu_element* eles, int32_t n_ele,
                           const bmadgpu_param* param, bmadgpu_lattice** out);
int bmadgpu_lattice_destroy(bmadgpu_lattice* lat);
/* Host-only validation and bookkeeping of an element list (no device needed): fills
 * n_step_out[n_ele] (nullable) with the resolved integration steps and *table_bytes (nullable)
 * with the packed table size. Returns BMADGPU_EUNSUPPORTED for elements off the device path. */
int bmadgpu_lattice_check(const bmadgpu_element* eles, int32_t n_ele, const bmadgpu_param* param,
                          int32_t* n_step_out, int64_t* table_bytes);
/* Resolved integration steps of element i (ds_step/num_steps bookkeeping); -1 on bad index. */
int32_t bmadgpu_lattice_n_step(const bmadgpu_lattice* lat, int32_t i);
/* Bytes of the packed element table (what is staged into shared memory). */
int64_t bmadgpu_lattice_table_bytes(const bmadgpu_lattice* lat);

/* ---- tracking ------------------------------------------------------------------------------- */
/* Track the bunch through elements [ix_start, ix_end) of the lattice, repeated over n_turns
 * turns, starting at turn index turn0. With ix_start = 0, ix_end = n_ele this is
 * n_turns passes of track_bunch(lat, bunch, ele0, ele0) as ltt_run_beam_mode does
 * (lt_tracking_mod.f90:1631-1713). Lost particles are skipped afterwards, as
 * track1_bunch_hom does (beam_utils.f90:83). Host buffers; copies in and out on ctx's stream.
 * moments: NULL, or [n_turns * BMADGPU_N_MOMENTS] sums over live particles after each turn. */
int bmadgpu_track_bunch(bmadgpu_ctx* ctx, const bmadgpu_lattice* lat, bmadgpu_bunch* bunch,
                        int32_t ix_start, int32_t ix_end, int32_t turn0, int32_t n_turns,
                        double* moments);

/* Same, with every pointer in the bunch (and moments) already in device memory; no copies. */
int bmadgpu_track_bunch_device(bmadgpu_ctx* ctx, const bmadgpu_lattice* lat, bmadgpu_bunch* bunch,
                               int32_t ix_start, int32_t ix_end, int32_t turn0, int32_t n_turns,
                               double* moments);

/* Largest bunch bmadgpu_track_bunch_device_noalloc accepts. */
#define BMADGPU_NOALLOC_MAX_PARTICLES 262144

/* No counterpart in the reference (an addition for callers that cannot allocate).
 * Same tracking as bmadgpu_track_bunch_device over the whole lattice (ix_start = 0,
 * ix_end = n_ele, no moments), with the live-particle list compacted every turns_per_launch
 * turns (0 = one launch), but allocating nothing: its scratch (two index lists and their
 * lengths, 2 MiB) is a fixed device array inside the library, for callers that cannot call
 * cudaMalloc mid-run: programs whose own pool allocator has taken the GPU's memory, and loops
 * that may not stall on an allocation (cudaMalloc can synchronise the device). Every bunch
 * pointer is device memory; the context and lattice already exist.
 * Limits: at most BMADGPU_NOALLOC_MAX_PARTICLES particles (BMADGPU_EINVAL otherwise). The
 * array is shared by all calls on a device and keeps the last call's contents (the lengths are
 * reset by each call); calls that overlap on the GPU race and must be serialised. The first
 * call on each device looks up the array's device address (cudaGetSymbolAddress) with that
 * device current: make that first call before any stream capture. The call only enqueues work on
 * the context's stream; a timed-out element-table staging wait inside it is reported by the next
 * bmadgpu_ctx_synchronize on the context (BMADGPU_ETIMEDOUT; the results are still correct). */
int bmadgpu_track_bunch_device_noalloc(bmadgpu_ctx* ctx, const bmadgpu_lattice* lat, bmadgpu_bunch* bunch,
                                       int32_t turn0, int32_t n_turns, int32_t turns_per_launch);

/* The per-element hook: one element for the whole bunch, the work of track1_bunch_hom
 * (beam_utils.f90:32-172) for bmad_standard elements. ix_ele is 0-based. */
int bmadgpu_track1_bunch(bmadgpu_ctx* ctx, const bmadgpu_lattice* lat, bmadgpu_bunch* bunch,
                         int32_t ix_ele, int32_t turn);

/* Waits for all work queued on the context's stream. */
int bmadgpu_ctx_synchronize(bmadgpu_ctx* ctx);

/* Launch shape of the tracking kernel, chosen by the autotuner or set by the caller. A new
 * context starts with {256, 2, 1, 0, 0}, the fastest shape measured on both a 451- and a
 * 1801-element ring. */
typedef struct bmadgpu_tuning {
  int32_t block;              /* threads per CTA: 64, 128, 256 or 512 */
  int32_t ctas_per_sm;        /* minimum resident CTAs per SM the register budget is compiled for
                                 (the variant with the largest such count not above it); 0 = the
                                 variant with the most registers per thread */
  int32_t stage_smem;         /* stage the element table in shared memory (TMA bulk copy); taken only
                                 when the copy leaves the resident CTAs per SM unchanged */
  int32_t turns_per_launch;   /* turns per kernel launch; 0 = all turns in one launch */
  int32_t compact;            /* compact the live-particle list between launches */
  int32_t reserved[3];
} bmadgpu_tuning;
int bmadgpu_ctx_set_tuning(bmadgpu_ctx* ctx, const bmadgpu_tuning* tuning);
int bmadgpu_ctx_get_tuning(const bmadgpu_ctx* ctx, bmadgpu_tuning* tuning);

/* Autotuner: times two one-turn trial launches of every launch shape (threads per CTA, register
 * budget via resident CTAs per SM, element table staged in shared memory or read through L1) on
 * a copy of the first min(n, sample_n) particles of a device-resident bunch (sample_n <= 0: 8192
 * per SM), sets the shape with the shortest trial as the context's tuning and returns it in
 * *chosen (nullable). The bunch is not modified. */
int bmadgpu_autotune(bmadgpu_ctx* ctx, const bmadgpu_lattice* lat, const bmadgpu_bunch* device_bunch,
                     int64_t sample_n, bmadgpu_tuning* chosen);

/* Device the context runs on, its SM count, and the CUDA stream it enqueues work on
 * (cudaStream_t, returned as void*). */
int bmadgpu_ctx_info(const bmadgpu_ctx* ctx, int32_t* device, int32_t* sm_count, void** stream);

/* Kernel launches this context has enqueued since it was created (all kernels of this library). */
int64_t bmadgpu_ctx_launch_count(const bmadgpu_ctx* ctx);

/* Measures the device's FP64 FMA throughput with a register-resident DFMA chain on every SM
 * (2 flops per FMA), a roofline denominator; *flops_per_s receives FLOP/s. */
int bmadgpu_measure_fp64_peak(bmadgpu_ctx* ctx, double* flops_per_s);

/* Self-check of the shared-reciprocal division the element maps use (a / b from RN(1/b) and one
 * FMA correction): *mismatches = how many of n pseudo-random pairs (seeded) differ in any bit from
 * the device's a / b. 0 is the only correct answer. */
int bmadgpu_selftest_division(bmadgpu_ctx* ctx, int64_t n, uint64_t seed, int64_t* mismatches);

/* The correctly rounded transcendentals the element maps use, evaluated on the device for n
 * arguments (device memory): fn 0 sin(a), 1 cos(a), 2 asin(a), 3 atan2(a, b), 4 sinh(a),
 * 5 cosh(a), 6 sincos(a) (sin in out[0, n), cos in out[n, 2n)), 7 sinhcosh(a) (likewise),
 * 8 exp(a), 9 tan(a). The reference calls its libm here (sin, cos, asin, atan2, sinh, cosh in
 * track_a_bend.f90:163-209, quad_mat2_calc.f90:34-47, track_a_rfcavity.f90:117; exp and tan in
 * the edge kicks of fringe_mod.f90); the device's are correctly rounded so that
 * its results equal the reference algorithm's with a correctly rounded libm, bit for bit. */
int bmadgpu_cr_eval(bmadgpu_ctx* ctx, int32_t fn, const double* a, const double* b, double* out, int64_t n);

/* sizeof() of the ABI structs as this library was compiled, for binding checks. */
int64_t bmadgpu_sizeof(int32_t which); /* 0 element, 1 param, 2 bunch, 3 tuning, 4 batch tuning,
                                           5 server config, 6 job info, 7 server stats,
                                           8 bunch data, 9 ltt params, 10 da params, 11 da point,
                                           12 twiss, 13 beam init, 14 fma params, 15 fma point */

/* ---- Batched tracking of many lattice variants -------------------------------------------
 * No single counterpart in the reference: it replaces a loop of long_term_tracking runs
 * (bsim/modules/lt_tracking_mod.f90:1571-1715, each a track_bunch per turn) over lattice
 * variants and dynamic-aperture grids (bmad/modules/dynamic_aperture_mod.f90:284-398), with
 * every variant's particles tracked in one persistent kernel launch per batch of turns.
 *
 * A batch holds n_var (lattice, particle count) pairs and owns the device particle state of
 * all of them: one structure-of-arrays block per variant, laid out one after another
 * (vec: variant v's [6][n_v] block follows variant v-1's; beta, t, state, ix_ele, ix_turn and
 * location likewise). Each launch hands out work items -- (variant, tile of live particles) --
 * from a device counter; CTAs stage the item's element table in shared memory when the variant
 * changes. Between launches the surviving particles of each variant are compacted (fused in the
 * tracking kernel: warp ballot + one atomic per warp). The launch sequence of a call is captured
 * once into a CUDA graph and replayed. Results per particle are bit-identical to
 * bmadgpu_track_bunch_device on the same variant with the same turns_per_launch. */
typedef struct bmadgpu_batch bmadgpu_batch;

typedef struct bmadgpu_batch_tuning {
  int32_t block;                /* threads per CTA: 64, 128, 256 or 512 */
  int32_t ctas_per_sm;          /* register budget as in bmadgpu_tuning (0 = most registers) */
  int32_t particles_per_thread; /* particles a thread tracks per work item: tile = block x this */
  int32_t turns_per_launch;     /* turns per launch, compaction in between; 0 = one launch */
  int32_t stage_smem;           /* stage each variant's element table in shared memory */
  int32_t use_graph;            /* replay each call's launch sequence as a CUDA graph */
  int32_t reserved[2];
} bmadgpu_batch_tuning;

/* counts[v] particles for lattices[v] (all lattices on the context's device; a lattice may
 * appear more than once). Device state starts zeroed. */
int bmadgpu_batch_create(bmadgpu_ctx* ctx, int32_t n_var, const bmadgpu_lattice* const* lattices,
                         const int64_t* counts, bmadgpu_batch** out);
int bmadgpu_batch_destroy(bmadgpu_batch* batch);
/* Device pointers of variant v's particles (v = -1: the whole batch, n = total count). */
int bmadgpu_batch_view(const bmadgpu_batch* batch, int32_t v, bmadgpu_bunch* device_view);
/* Copies variant v (v = -1: all variants, in the batch layout) from host memory; enqueued on the
 * context stream, so the host buffers must stay valid until the next synchronisation. Fields
 * passed as NULL (t, ix_ele, ix_turn, location) are left as they are on the device. */
int bmadgpu_batch_upload(bmadgpu_batch* batch, int32_t v, const bmadgpu_bunch* host);
/* Copies variant v (v = -1: all) to host memory and waits for it. */
int bmadgpu_batch_download(bmadgpu_batch* batch, int32_t v, bmadgpu_bunch* host);
/* Tracks every variant's live particles through its whole lattice for n_turns turns numbered
 * from turn0; enqueued on the context stream (bmadgpu_ctx_synchronize waits and reports a
 * staging time-out). */
int bmadgpu_batch_track(bmadgpu_batch* batch, int32_t turn0, int32_t n_turns);
int bmadgpu_batch_set_tuning(bmadgpu_batch* batch, const bmadgpu_batch_tuning* tuning);
int bmadgpu_batch_get_tuning(const bmadgpu_batch* batch, bmadgpu_batch_tuning* tuning);
/* Autotuner: times trial calls of sample_turns turns (0: 8) for every launch shape, then
 * particles per thread, then turns per launch, on the batch's current state, which it restores
 * after each trial; sets the fastest and returns it in *chosen (nullable). */
int bmadgpu_batch_autotune(bmadgpu_batch* batch, int32_t sample_turns, bmadgpu_batch_tuning* chosen);

/* ---- Serving: continuous batching of tracking jobs -----------------------------------------
 * No counterpart in the reference: it serves the jobs that Bmad programs run one at a time --
 * long_term_tracking bunch runs (bsim/modules/lt_tracking_mod.f90:1571-1715), dynamic-aperture
 * scans (bmad/modules/dynamic_aperture_mod.f90:284-398), frequency-map grids
 * (bsim/frequency_map/frequency_map.f90:183-330) -- as requests arriving at any time.
 *
 * A server owns a resident particle arena in device memory, sized at creation from the free HBM,
 * and a worker thread. Submitted jobs wait in a queue; the worker admits them (shortest remaining
 * work first, or in arrival order) while job slots, arena space and the live-particle target
 * allow, uploads their particles on a copy stream while the current round runs, and runs rounds:
 * one persistent batched launch in which every resident job advances max(1, element_steps /
 * n_ele) turns (the batched kernel, with fused compaction). Jobs finished after a round are
 * copied back into the caller's host arrays on the copy stream, overlapping the next round, and
 * their slot and arena space go to waiting jobs. Lattice tables stay resident (the caller's
 * lattice objects must outlive the jobs that use them). A job's result is bit-identical to the
 * plain path run alone with turns_per_launch equal to the job's turns per round. */
typedef struct bmadgpu_server bmadgpu_server;

enum { BMADGPU_SERVE_SRPT = 0, BMADGPU_SERVE_FIFO = 1 };
enum { BMADGPU_JOB_QUEUED = 0, BMADGPU_JOB_RUNNING = 1, BMADGPU_JOB_DONE = 2, BMADGPU_JOB_CANCELLED = 3 };

typedef struct bmadgpu_server_config {
  int64_t max_particles;   /* resident particle capacity; 0 = hbm_fraction of the free device memory */
  double hbm_fraction;     /* share of free device memory the arena may take (0: 0.5) */
  int32_t max_jobs;        /* jobs resident at once (0: 4096) */
  int32_t element_steps;   /* element passes per particle per round (0: 4096) */
  int64_t target_live;     /* no admission while this many live particles are resident (0: 1,048,576) */
  int32_t policy;          /* BMADGPU_SERVE_SRPT or BMADGPU_SERVE_FIFO */
  int32_t block;           /* round kernel shape as bmadgpu_batch_tuning (0: 128) */
  int32_t ctas_per_sm;     /* (0 with block 0: 4) */
  int32_t stage_smem;      /* stage element tables of up to 64 KiB in shared memory */
  int32_t record_mib;      /* record arena of frequency-map jobs in MiB (0: a quarter of the device
                              memory still free after the particle arena) */
  int32_t reserved[3];
} bmadgpu_server_config;

typedef struct bmadgpu_job_info {
  int32_t status;          /* BMADGPU_JOB_* */
  int32_t rounds;          /* rounds the job took part in */
  double t_submit, t_admit, t_done;  /* seconds on the server's clock (-1 when not reached) */
  int64_t particle_turns;  /* turns tracked summed over particles (lost ones up to their loss) */
} bmadgpu_job_info;

typedef struct bmadgpu_server_stats {
  int64_t jobs_submitted, jobs_done, rounds, particle_turns;
  double elapsed_s;        /* first submission to the last completion */
  double latency_p50_s, latency_p99_s, latency_max_s;  /* t_done - t_submit over finished jobs */
  int64_t capacity;        /* resident particle capacity */
  int64_t peak_resident;   /* most particles resident at once */
  /* the compute stream's timeline over the completed rounds (first round's start to the last
   * one's end): time inside rounds, the sum of the gaps between consecutive rounds (the stream
   * waiting for the worker's admission and bookkeeping, or for work), and the longest gap */
  double gpu_busy_s, gpu_idle_s, gpu_max_gap_s;
} bmadgpu_server_stats;

/* cfg may be NULL (all defaults). The server runs on the context's device with its own streams. */
int bmadgpu_server_create(bmadgpu_ctx* ctx, const bmadgpu_server_config* cfg, bmadgpu_server** out);
/* Cancels queued jobs, lets resident ones finish, stops the worker and frees the server. */
int bmadgpu_server_destroy(bmadgpu_server* server);
/* Queues a job: the bunch (host memory; pinned memory from bmadgpu_host_alloc lets its copies
 * overlap with tracking) is tracked through the whole lattice for n_turns turns numbered from
 * turn0 and written back in place. The bunch arrays must stay valid and untouched until the job is
 * done. BMADGPU_ENOMEM if the bunch can never fit the arena, BMADGPU_EBUSY if the queue is full. */
int bmadgpu_server_submit(bmadgpu_server* server, const bmadgpu_lattice* lat, bmadgpu_bunch* bunch, int32_t turn0,
                          int32_t n_turns, int64_t* job_id);
/* A frequency-map job (frequency_map.f90:197-376 for these particles): bunch holds the start
 * coordinates (closed orbit + grid offsets), tracked n_turns turns like any job, while every turn's
 * normalised coordinates are recorded on the device (params: normalisation, closed orbit, z_cut,
 * fft_turns, ring tunes; params->n_turn is not used). When the job completes, points [n] hold each
 * particle's tunes or its status as bmadgpu_fma gives them, and the bunch arrays its final
 * coordinates. The record (48 B per particle-turn) comes from the server's record arena. */
struct bmadgpu_fma_params;
struct bmadgpu_fma_point;
int bmadgpu_server_submit_fma(bmadgpu_server* server, const bmadgpu_lattice* lat, bmadgpu_bunch* bunch, int32_t turn0,
                              int32_t n_turns, const struct bmadgpu_fma_params* params,
                              struct bmadgpu_fma_point* points, int64_t* job_id);
int bmadgpu_server_job(bmadgpu_server* server, int64_t job_id, bmadgpu_job_info* info);
/* Waits until the job (job_id = -1: every submitted job) is done or cancelled; BMADGPU_ETIMEDOUT
 * after timeout_s seconds. Also reports an error the worker met. */
int bmadgpu_server_wait(bmadgpu_server* server, int64_t job_id, double timeout_s);
int bmadgpu_server_get_stats(bmadgpu_server* server, bmadgpu_server_stats* stats);

/* ---- Differentiation ------------------------------------------------------------------------
 * No counterpart in the reference, which has no derivative of tracking with respect to element
 * strengths other than Tao's one-sided finite differences (tao/code/tao_dmerit_mod.f90:162-180).
 *
 * loss = (1/n) sum over the particles still alive after n_turns of (x^2 + y^2), tracking the host
 * bunch (vec, beta, state; left unchanged) through the whole lattice from turn 0. grad[i] =
 * d(loss)/d(k) for element param_ele[i] (0-based): k1 of a quadrupole, k2 of a sextupole, k3 of
 * an octupole; the element's strength must be non-zero and its other field coefficients must scale
 * with it (no hkick/vkick; multipoles only with scale_multipoles). Computed by a hand-written
 * adjoint of the element maps, one thread per particle, with a checkpoint every checkpoint_every
 * turns and recomputation in between. Lattices with edge fringe, bends with k1 or multipoles,
 * thin multipoles, pitched or offset bends, electric multipoles or elements of more than 16 steps
 * give BMADGPU_EUNSUPPORTED. Lost particles
 * leave the loss (the set of survivors is held fixed). */
int bmadgpu_loss_grad(bmadgpu_ctx* ctx, const bmadgpu_lattice* lat, const bmadgpu_bunch* host_bunch, int32_t n_turns,
                      int32_t checkpoint_every, int32_t n_param, const int32_t* param_ele, double* loss,
                      double* grad);

/* ---- Long-term tracking outputs ------------------------------------------------------------
 * Bunch data of ltt_calc_bunch_data / calc_bunch_params (bsim/modules/lt_tracking_mod.f90:
 * 2369-2451, bmad/multiparticle/beam_utils.f90:1326-1690) over the live particles. */
typedef struct bmadgpu_bunch_data {
  int64_t n_live;
  double t, sigma_t, p0c;       /* <t>, rms t, reference momentum */
  double centroid[6];           /* <vec> */
  double sigma_vec[21];         /* <v_i v_j> - <v_i><v_j>, i <= j, with the round-off zeroing rule (ltt .sigma) */
  double sig1[6];               /* sqrt of its diagonal */
  double skew[3], kurt[3];      /* x, y, z: <d^3>/sig^3 and <d^4>/sig^4 - 3 (n_live >= 10) */
  double sigma[36];             /* centred sigma matrix <(v - <v>)(v - <v>)^T> */
  double emit[3], norm_emit[3]; /* normal-mode a, b, c emittances (eigenvalues of sigma.S), n_live >= 6 */
  double proj_emit[3], proj_beta[3], proj_alpha[3];  /* projected x, y, z (dispersion removed) */
  double eta[2], etap[2];       /* x, y dispersion from the sigma matrix */
  int32_t emit_valid;           /* 1 if the normal-mode analysis succeeded */
  int32_t reserved;
} bmadgpu_bunch_data;

/* Bunch data of a device-resident bunch (two-pass device sums, deterministic reduction order). */
int bmadgpu_bunch_stats(bmadgpu_ctx* ctx, const bmadgpu_lattice* lat, const bmadgpu_bunch* device_bunch,
                        bmadgpu_bunch_data* data);
/* Host-only: bunch data from the 63 sums of the two passes (count, sum v, sum t, sum t^2,
 * sum v_i v_j; centred sum d_i d_j, sum d^3, sum d^4), for callers with their own sums. */
int bmadgpu_bunch_data_from_sums(const double* sums, double p0c, double mass, bmadgpu_bunch_data* data);
/* Host only: the normal-mode emittances emit [3] (nullable) and the normal-form matrix n_mat [36]
 * (row-major; sigma = N diag(emit) N^T up to Q's single-precision entries) of a 6x6 sigma matrix, as
 * calc_emittances_and_twiss_from_sigma_matrix returns them in n_mat
 * (bmad/multiparticle/beam_utils.f90:1495-1551). BMADGPU_EINVAL if sigma is not positive definite. */
int bmadgpu_sigma_normal_form(const double* sigma, double* emit, double* n_mat);

/* ltt_run_beam_mode (lt_tracking_mod.f90:1571-1715) for one bunch with bmad_standard tracking:
 * turns ix_turn_start .. n_turns - 1 with the reference's stop conditions (no particle left; lost count reaching
 * nint(dead_cutoff * n)), writing the averages files (<averages_file>.ave / .sigma / .emit, the
 * reference's columns and number formats) and phase-space files (<phase_space_file> with the turn
 * number, zero-padded, appended or put in place of '#'). Output schedules as the reference's
 * *_output_every_n_turns: -1 last turn only, 0 first and last turn, n > 0 every n turns. The host
 * bunch is updated to the final state; *turns_done receives the turns tracked. */
typedef struct bmadgpu_ltt_params {
  int32_t n_turns;
  int32_t averages_every_n_turns;
  int32_t particle_every_n_turns;
  int32_t output_only_last_turns;   /* > 0: outputs only within the last this-many turns */
  int32_t only_live_particles_out;  /* phase-space files list only live particles */
  int32_t ix_turn_start;            /* turn number of the bunch as given (resume from a beam file) */
  int32_t beam_every_n_turns;       /* beam files every n turns (and at n_turns); -1: at n_turns only */
  int32_t beam_exact;               /* beam files with 17 digits and beta (bit-exact resume) */
  double dead_cutoff;               /* 0 means 1 (the reference default) */
  const char* averages_file;        /* NULL or "": no averages output */
  const char* phase_space_file;     /* NULL or "": no phase-space output */
  const char* beam_file;            /* NULL or "": no beam files; "<stem>-<turn><.ext>" as ltt_write_beam_file names them */
  double core_emit_cutoff[8];       /* ltt%core_emit_cutoff: core fractions whose emittances the .emit file adds,
                                       up to the first entry <= 0; all zero: the reference's default, 0.5;
                                       core_emit_cutoff[0] < 0: none */
  int32_t core_emit_per_mode;       /* .not. ltt%core_emit_combined_calc: a core per normal mode, ranked by
                                       that mode's action (0: the combined calculation, the default) */
  const char* action_angle_file;    /* ltt%action_angle_output_file: NULL or "": none; written with the
                                       phase-space schedule, actions and angles about the bunch's own
                                       normal form (calc_bunch_params' n_mat) */
  const char* per_particle_file;    /* ltt%per_particle_output_file: NULL or "": none; one file per
                                       particle (at most 1000 particles, as the reference requires) */
  const double* action_angle_n_inv; /* [36] row-major or NULL: with ltt%action_angle_calc_uses_1turn_matrix
                                       the caller's N^-1 of the one-turn matrix (make_N,
                                       bmad/modules/mode3_mod.f90:825-912, then mat_inverse); the
                                       actions are then taken about zero, as the reference's
                                       write_this_data does (lt_tracking_mod.f90:2007-2022) */
} bmadgpu_ltt_params;
int bmadgpu_ltt_run(bmadgpu_ctx* ctx, const bmadgpu_lattice* lat, bmadgpu_bunch* host_bunch,
                    const bmadgpu_ltt_params* params, int32_t* turns_done);
/* Core emittances a, b, c of a device-resident bunch for one core fraction cutoff (0, 1] as
 * ltt_calc_bunch_data computes them (bsim/modules/lt_tracking_mod.f90:2432-2516): combined_calc != 0
 * ranks by the combined normalised amplitude (ltt%core_emit_combined_calc, the default), 0 gives
 * each mode its own core ranked by that mode's action; zeros where the reference leaves them zero
 * (fewer than 10 live particles, a zero bunch emittance, an empty core). */
int bmadgpu_bunch_core_emit(bmadgpu_ctx* ctx, const bmadgpu_lattice* lat, const bmadgpu_bunch* device_bunch,
                            double cutoff, int32_t combined_calc, double* core_emit);

/* The core selection used by bmadgpu_bunch_core_emit and the LTT core emittances: of n
 * non-negative amplitudes (device memory), the n_cut smallest, ties going to the lower index as
 * the reference's stable sort ranks them (bsim/modules/lt_tracking_mod.f90:2550). mask (device, [n])
 * gets BMADGPU_ALIVE for the selected and 0 for the others. Amplitudes of 1e99 and above,
 * infinite and NaN amplitudes mark particles that cannot be in a core: if the n_cut-th smallest
 * is one of them, *selected = 0 and mask is left as it was; otherwise *selected = 1. */
int bmadgpu_select_smallest(bmadgpu_ctx* ctx, const double* keys, int64_t n, int64_t n_cut, int32_t* mask,
                            int32_t* selected);

/* ---- Dynamic aperture ------------------------------------------------------------------------
 * dynamic_aperture_point (bmad/modules/dynamic_aperture_mod.f90:284-398) for many rays at once:
 * along the ray (x, y) = (cos theta x_init, sin theta y_init) s, starting at s = 1, a trial
 * particle (start orbit + (x, 0, y, 0, 0, 0)) is tracked n_turn turns; survival doubles s until a
 * loss brackets the aperture, then the bracket is halved until it is within
 * 2 (abs_accuracy + r rel_accuracy). Every iteration tracks the trial particles of all unfinished
 * rays in one launch and updates the searches on the device. */
typedef struct bmadgpu_da_params {
  double x_init, y_init;            /* aperture_param%x_init, %y_init [m] */
  double abs_accuracy, rel_accuracy;
  int32_t n_turn;
  int32_t max_iterations;           /* per ray (0: 200); the reference loops without limit */
} bmadgpu_da_params;
typedef struct bmadgpu_da_point {
  double x, y;                      /* the aperture point relative to the start orbit */
  int32_t i_turn;                   /* turn of the last loss (counted from 1, as the reference) */
  int32_t ix_ele;                   /* element of that loss (0-based) */
  int32_t plane;                    /* its state code (lost_neg_x, ...) */
  int32_t iterations;
} bmadgpu_da_point;
/* orb0: [n_rays][6] start orbits (e.g. closed orbit, or an energy offset per ray), or NULL for
 * zero. BMADGPU_ETIMEDOUT if a ray reached 1 m or the iteration limit (its point is still set). */
int bmadgpu_da_scan(bmadgpu_ctx* ctx, const bmadgpu_lattice* lat, int32_t n_rays, const double* theta,
                    const double* orb0, const bmadgpu_da_params* params, bmadgpu_da_point* points);

/* ---- Optics: closed orbit, one-turn matrix, periodic Twiss, matched beam ---------------------
 * What long_term_tracking computes before it tracks (twiss_and_track, lt_tracking_mod.f90:562,
 * and ltt_init_beam_distribution, lt_tracking_mod.f90:1548-1561). Matrices are 6x6 row-major:
 * mat[i*6 + j] = Fortran mat6(i+1, j+1). */

/* One-turn matrix about `orbit` [6] by fourth-order central differences of one turn of device
 * tracking (25 particles in one launch), apertures off; rf_on = 0 tracks every rfcavity as
 * switched off (the matrix twiss_at_start.f90:29 uses). orbit_end [6] (nullable) receives the
 * tracked orbit. Replaces transfer_matrix_calc after lat_make_mat6 (closed_orbit_calc.f90:787-788). */
int bmadgpu_one_turn_matrix(bmadgpu_ctx* ctx, const bmadgpu_lattice* lat, const double* orbit, int32_t rf_on,
                            double* orbit_end, double* mat);
/* Closed orbit at the lattice start (closed_orbit_calc, closed_orbit_calc.f90:192-862), forward
 * direction. dim = 4: transverse at the fixed pz = orbit[5], RF off, z starts at 0; 5: RF off,
 * pz adjusted until z closes; 6: full 6D with RF on; 0: 6 if any cavity is on, else 4. orbit [6]
 * is the initial guess in and the closed orbit out; mat [36] (nullable) receives the one-turn
 * matrix there. Stops when |f(x)_i - x_i| < |x_i| rel_tol + abs_tol for the fitted coordinates
 * (<= 0: bmad_com's 1e-9 and 1e-12); max_iter <= 0: 100. BMADGPU_ETIMEDOUT if not converged. */
int bmadgpu_closed_orbit(bmadgpu_ctx* ctx, const bmadgpu_lattice* lat, int32_t dim, double* orbit, double* mat,
                         double rel_tol, double abs_tol, int32_t max_iter, int32_t* iterations);

/* Status codes of the Twiss calculation (matrix_status, bmad_struct.f90:186-187). */
enum {
  BMADGPU_TWISS_OK = 1, BMADGPU_TWISS_IN_STOP_BAND = 2, BMADGPU_TWISS_NON_SYMPLECTIC = 3,
  BMADGPU_TWISS_UNSTABLE = 4, BMADGPU_TWISS_UNSTABLE_A = 5, BMADGPU_TWISS_UNSTABLE_B = 6
};
/* ele%a, ele%b, ele%x, ele%y, ele%c_mat, ele%gamma_c as twiss_from_mat6 fills them. phi_a/phi_b
 * are the one-turn phase advances in [0, 2 pi) (the tunes times 2 pi). */
typedef struct bmadgpu_twiss {
  double beta_a, alpha_a, gamma_a, phi_a;
  double beta_b, alpha_b, gamma_b, phi_b;
  double eta_a, etap_a, deta_ds_a, eta_b, etap_b, deta_ds_b;   /* normal-mode dispersion */
  double eta_x, etap_x, deta_ds_x, eta_y, etap_y, deta_ds_y;   /* lab-frame dispersion */
  double c_mat[4];            /* c_mat(1,1), (1,2), (2,1), (2,2) */
  double gamma_c;
  double growth_rate;         /* when not stable */
  double symp_error;          /* mat_symp_error of the 4x4 block */
  int32_t status;             /* BMADGPU_TWISS_* */
  int32_t reserved;
} bmadgpu_twiss;
/* Periodic Twiss from a one-turn matrix (twiss_from_mat6.f90:24, mat_symp_decouple.f90:22,
 * twiss_from_mat2.f90:19); orb0 [6] (nullable) is the orbit for the deta_ds terms. Host-only.
 * Returns BMADGPU_OK with tw->status telling whether the optics are stable. */
int bmadgpu_twiss_from_mat6(const double* mat, const double* orb0, bmadgpu_twiss* tw);

/* beam_init_struct fields of a Gaussian bunch (beam_init_struct, bmad_struct.f90). */
typedef struct bmadgpu_beam_init {
  double a_emit, b_emit;      /* geometric emittances [m] */
  double sig_z, sig_pz;
  double dpz_dz;
  double sig_z_jitter, sig_pz_jitter;
  double center[6];
  double center_jitter[6];
  double sigma_cutoff;        /* random_sigma_cutoff: <= 0 none */
  uint64_t seed;              /* Philox4x32-10 key */
  int32_t renorm_center;
  int32_t renorm_sigma;
} bmadgpu_beam_init;
/* Fills the device bunch (n = bunch->n particles) with a Gaussian beam matched to tw
 * (init_bunch_distribution with RAN_GAUSS in all planes, beam_utils.f90:328-535, 551-721), plus
 * orbit [6] (nullable) as add_closed_orbit_to_init_position adds it. Deviates: normals (device,
 * nullable) = [6*n] SoA per particle, then the sig_z and sig_pz jitters, then the 6 centre jitters
 * ([6*n + 8] in all); NULL draws them on the device from a counter-based Philox4x32-10 stream keyed
 * by bi->seed (deviate k of particle i from counter (i, attempt, k)). */
int bmadgpu_beam_init_gaussian(bmadgpu_ctx* ctx, const bmadgpu_param* param, const bmadgpu_twiss* tw,
                               const bmadgpu_beam_init* bi, const double* normals, const double* orbit,
                               bmadgpu_bunch* device_bunch);
/* The deviates bmadgpu_beam_init_gaussian draws for (seed, sigma_cutoff, n): d_out [6*n + 8] (device). */
int bmadgpu_gaussian_deviates(bmadgpu_ctx* ctx, uint64_t seed, double sigma_cutoff, int64_t n, double* d_out);
/* The Philox4x32-10 block function those deviates come from (host-only): out = philox(counter [4], key [2]). */
int bmadgpu_philox4x32_10(const uint32_t* counter, const uint32_t* key, uint32_t* out);

/* ---- Frequency-map analysis -----------------------------------------------------------------
 * frequency_map (bsim/frequency_map/frequency_map.f90:197-376) for all particles at once: start at
 * orbit + offset, n_turn turns of tracking with the normalised coordinates recorded every turn, then
 * per particle the Hanning-windowed spectra of x + i px, y + i py, z - i pz over the first and the
 * last fft_turns turns and calc_tune's interpolated peak (frequency_map.f90:364-375). */
typedef struct bmadgpu_fma_params {
  int32_t n_turn;
  int32_t fft_turns;          /* 0: n_turn / 2 (at most 4096) */
  int32_t z_cut;              /* stop a particle whose |z - z_co| exceeds a quarter RF wavelength */
  int32_t reserved;
  double rf_frequency;        /* for z_cut; <= 0: the lowest frequency of the lattice's cavities */
  double norm[36];            /* psv_norm = norm (vec - orbit), row-major: V^-1 (uncoupled RF-off
                                 matrix) or Tinv^T from the eigenvectors, as the reference chooses */
  double orbit[6];            /* closed orbit co(0) */
  double tune_a, tune_b;      /* ring tunes phi/2pi: below 0.5 the x/y results are 1 - Q as there */
} bmadgpu_fma_params;
typedef struct bmadgpu_fma_point {
  double tune[6];             /* Qx0, Qy0, Qz0 (first fft_turns turns), Qx1, Qy1, Qz1 (last) */
  int32_t status;             /* 0 tunes computed, 1 lost, 2 outside the RF bucket */
  int32_t turn_lost;          /* turn (from 1) where status was set */
  int32_t ix_ele;             /* element of the loss (0-based), status 1 */
  int32_t reserved;
} bmadgpu_fma_point;
/* offsets: [n_particles][6] start offsets from the closed orbit. */
int bmadgpu_fma(bmadgpu_ctx* ctx, const bmadgpu_lattice* lat, int32_t n_particles, const double* offsets,
                const bmadgpu_fma_params* params, bmadgpu_fma_point* points);
/* The reference's .fm table for these particles (host-only): header unless append, then
 * '(12e14.5)' rows, '*' tune columns for status 2, no row for lost particles. */
int bmadgpu_fma_write(const char* path, int32_t n_particles, const double* offsets,
                      const bmadgpu_fma_point* points, int32_t append);

/* NAFF frequency decomposition (naff, sim_utils/math/naff.f90:72-131) of n_signals complex
 * signals of n_samples points each (4..4096; any length): cdata [n_signals][n_samples] as
 * interleaved (re, im) doubles, Fortran complex(rp) layout, in host memory. Per signal n_comp
 * components: freqs [n_signals][n_comp] in units of 2 pi (data ~ amp exp(-2 pi i f t)), amps
 * [n_signals][n_comp] interleaved complex. zero_first: the first component is f = 0. As in the
 * reference, a signal whose points are all equal gets freqs 0, and a failed peak estimate leaves
 * the remaining freqs at -1. One CTA per signal on the device. */
int bmadgpu_naff(bmadgpu_ctx* ctx, int32_t n_signals, int32_t n_samples, const double* cdata, int32_t n_comp,
                 int32_t zero_first, double* freqs, double* amps);

/* ---- Beam files (checkpoint / resume) -------------------------------------------------------
 * Bmad's ASCII beam file, version 4 (write_ascii_beam_file / read_beam_ascii,
 * bmad/multiparticle/beam_file_io.f90:112-300, 834-1282). Host-only; no GPU needed. */
enum { BMADGPU_BEAM_ALIVE_ONLY = 1, BMADGPU_BEAM_APPEND = 2, BMADGPU_BEAM_EXACT = 4, BMADGPU_BEAM_AT_ELEMENT = 8 };
/* Writes one bunch; flags: ALIVE_ONLY (skip lost particles), APPEND, EXACT (17 significant
 * digits and a beta column, so a resumed run continues bit for bit; otherwise the reference's
 * es23.15). ix_ele is written 1-based as Bmad numbers elements (0 for particles not lost). */
int bmadgpu_beam_write_ascii(const char* path, const bmadgpu_bunch* host_bunch, const bmadgpu_param* param,
                             double s_position, int32_t flags);
/* Reads a file written as above (or by Bmad): with host_bunch NULL or host_bunch->vec NULL only
 * *n_particle is set; otherwise host_bunch->n must equal it and the arrays are filled (beta from
 * the file's beta column, else from pz as init_coord computes it). */
int bmadgpu_beam_read_ascii(const char* path, const bmadgpu_param* param, bmadgpu_bunch* host_bunch,
                            int64_t* n_particle);

/* Bmad's openPMD beam file in HDF5 (hdf5_write_beam, bmad/hdf5/hdf5_write_beam.f90:20-245), written
 * without the HDF5 library in the classic file structures libhdf5 writes by default. One bunch as
 * /data/00001/particles/<species>/; records whose values are all equal become constant record
 * components, as in the reference. flags: ALIVE_ONLY; APPEND (to a file whose basePath is
 * "/data/%T/": its objects are copied, lastUpdated is stamped and the bunch takes the first free
 * number; files with shared datatypes give BMADGPU_EUNSUPPORTED). The
 * species name comes from param's mass and charge (electron, positron, proton, anti-proton;
 * other species give BMADGPU_EUNSUPPORTED). Spin and macro-charge are written as 0. */
int bmadgpu_beam_write_hdf5(const char* path, const bmadgpu_bunch* host_bunch, const bmadgpu_param* param,
                            double s_position, int32_t flags);
/* The same for n_bunch bunches (1 to 256) of one species in one file, /data/00001/ to /data/<n>/,
 * as hdf5_write_beam writes bunches(:). */
int bmadgpu_beam_write_hdf5_bunches(const char* path, const bmadgpu_bunch* host_bunches, int32_t n_bunch,
                                    const bmadgpu_param* param, double s_position, int32_t flags);
/* hdf5_read_beam (bmad/hdf5/hdf5_read_beam.f90:24-474) without an element: bunch ix_bunch
 * (0-based, in the order of the bunch groups' names) of a file written by Bmad or by the call above,
 * the old layout (records directly in particles/) included. *n_bunch (nullable) is set to the
 * number of bunches and *n_particle to the bunch's size; with host_bunch NULL or host_bunch->vec
 * NULL nothing else is read, otherwise host_bunch->n must equal *n_particle. beta comes from the
 * momentum and param's mass. Files using HDF5 structures outside the classic set (superblock
 * version 2 or 3, version-2 object headers, link messages, chunked or filtered storage) and photon
 * bunches give BMADGPU_EUNSUPPORTED. flags: BMADGPU_BEAM_AT_ELEMENT reads as the reference does when
 * given the lattice's beginning element (as long_term_tracking reads its starting beam): px and py
 * are divided by param's p0c, beta follows from it, and every particle is placed at the exit of
 * the beginning element (ix_ele -1, downstream_end); pz stays relative to the file's p0c. */
int bmadgpu_beam_read_hdf5(const char* path, const bmadgpu_param* param, int32_t ix_bunch, int32_t flags,
                           bmadgpu_bunch* host_bunch, int64_t* n_particle, int32_t* n_bunch);
/* write_beam_file / read_beam_file (bmad/multiparticle/beam_file_io.f90:29-106, 380-420): HDF5
 * (the two calls above; the first bunch on reading) when the name ends in ".h5" or ".hdf5", else
 * the ASCII calls. The long-term-tracking beam files go through the writer. */
int bmadgpu_beam_write_file(const char* path, const bmadgpu_bunch* host_bunch, const bmadgpu_param* param,
                            double s_position, int32_t flags);
int bmadgpu_beam_read_file(const char* path, const bmadgpu_param* param, bmadgpu_bunch* host_bunch,
                           int64_t* n_particle);

/* Page-locked host memory for bunch arrays (cudaHostAlloc / cudaFreeHost). */
int bmadgpu_host_alloc(int64_t bytes, void** ptr);
int bmadgpu_host_free(void* ptr);


#ifdef __cplusplus
}
#endif

#endif /* BMADGPU_H */
