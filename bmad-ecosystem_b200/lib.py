"""ctypes binding of libbmadgpu.so (include/bmadgpu.h) and a thin object layer over it.

Names follow the reference: ``track_bunch`` is track_bunch (bmad/multiparticle/beam_mod.f90:103)
over turns, ``track1_bunch`` the per-element hook (beam_mod.f90:238). Errors raise
``BmadGpuError`` with the library's last-error message; nothing here falls back to a CPU path.

Two builds of the library share this binding: libbmadgpu.so (the device libm in the element
maps, the default) and libbmadgpu_cr.so (correctly rounded transcendentals: bit-identical to the
reference's algorithm run with a correctly rounded libm). ``set_math("cr")`` (or the environment
variable BMADGPU_MATH=cr) selects the second for everything created afterwards; an object keeps
calling the build that was current when it was made only if the selection is not changed while
it lives.
"""
import ctypes as C
import math
import os
import re

import numpy as np

from . import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libbmadgpu.so")
LIB_CR_PATH = os.path.join(_HERE, "lib", "libbmadgpu_cr.so")
MATH = ("fast", "cr")
HEADER_PATH = os.path.join(os.path.dirname(_HERE), "include", "bmadgpu.h")


class BmadGpuError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s (%d): %s" % (abi.STATUS_NAMES.get(code, "?"), code, msg))
        self.code = code


class Tuning(C.Structure):
    _fields_ = [("block", C.c_int32), ("ctas_per_sm", C.c_int32), ("stage_smem", C.c_int32),
                ("turns_per_launch", C.c_int32), ("compact", C.c_int32), ("reserved", C.c_int32 * 3)]


class BatchTuning(C.Structure):
    _fields_ = [("block", C.c_int32), ("ctas_per_sm", C.c_int32), ("particles_per_thread", C.c_int32),
                ("turns_per_launch", C.c_int32), ("stage_smem", C.c_int32), ("use_graph", C.c_int32),
                ("reserved", C.c_int32 * 2)]


_BATCH_FIELDS = ("block", "ctas_per_sm", "particles_per_thread", "turns_per_launch", "stage_smem", "use_graph")

_libs = {}
_math = os.environ.get("BMADGPU_MATH", "fast")


def set_math(math):
    """Select the library build for what is created from now on: "fast" (libbmadgpu.so) or "cr"
    (libbmadgpu_cr.so, correctly rounded transcendentals)."""
    global _math
    if math not in MATH:
        raise BmadGpuError(abi.EINVAL, "math must be one of %s" % (MATH,))
    _math = math


def get_math():
    return _math


def load(path=None):
    """Load the shared library of the selected build (built by csrc/Makefile; BMADGPU_LIBRARY and
    BMADGPU_LIBRARY_CR override the paths). Raises if it is missing."""
    if path is None:
        if _math == "cr":
            path = os.environ.get("BMADGPU_LIBRARY_CR") or LIB_CR_PATH
        else:
            path = os.environ.get("BMADGPU_LIBRARY") or LIB_PATH
    if path in _libs:
        return _libs[path]
    if not os.path.exists(path):
        raise BmadGpuError(abi.EINVAL, "%s not built: run make -C bmad-ecosystem_b200/csrc" % os.path.basename(path))
    lib = C.CDLL(path)
    P, V = C.POINTER, C.c_void_p
    sig = {
        "bmadgpu_abi_version": ([], C.c_int),
        "bmadgpu_last_error": ([], C.c_char_p),
        "bmadgpu_sizeof": ([C.c_int32], C.c_int64),
        "bmadgpu_ctx_create": ([C.c_int32, P(V)], C.c_int),
        "bmadgpu_ctx_destroy": ([V], C.c_int),
        "bmadgpu_ctx_synchronize": ([V], C.c_int),
        "bmadgpu_ctx_set_tuning": ([V, P(Tuning)], C.c_int),
        "bmadgpu_ctx_get_tuning": ([V, P(Tuning)], C.c_int),
        "bmadgpu_ctx_info": ([V, P(C.c_int32), P(C.c_int32), P(V)], C.c_int),
        "bmadgpu_lattice_create": ([V, P(abi.Element), C.c_int32, P(abi.Param), P(V)], C.c_int),
        "bmadgpu_lattice_destroy": ([V], C.c_int),
        "bmadgpu_lattice_n_step": ([V, C.c_int32], C.c_int32),
        "bmadgpu_lattice_table_bytes": ([V], C.c_int64),
        "bmadgpu_lattice_check": ([P(abi.Element), C.c_int32, P(abi.Param), P(C.c_int32), P(C.c_int64)], C.c_int),
        "bmadgpu_track_bunch": ([V, V, P(abi.Bunch), C.c_int32, C.c_int32, C.c_int32, C.c_int32, V], C.c_int),
        "bmadgpu_track_bunch_device": ([V, V, P(abi.Bunch), C.c_int32, C.c_int32, C.c_int32, C.c_int32, V],
                                       C.c_int),
        "bmadgpu_track1_bunch": ([V, V, P(abi.Bunch), C.c_int32, C.c_int32], C.c_int),
        "bmadgpu_ctx_launch_count": ([V], C.c_int64),
        "bmadgpu_measure_fp64_peak": ([V, P(C.c_double)], C.c_int),
        "bmadgpu_autotune": ([V, V, P(abi.Bunch), C.c_int64, P(Tuning)], C.c_int),
        "bmadgpu_batch_create": ([V, C.c_int32, P(V), P(C.c_int64), P(V)], C.c_int),
        "bmadgpu_batch_destroy": ([V], C.c_int),
        "bmadgpu_batch_view": ([V, C.c_int32, P(abi.Bunch)], C.c_int),
        "bmadgpu_batch_upload": ([V, C.c_int32, P(abi.Bunch)], C.c_int),
        "bmadgpu_batch_download": ([V, C.c_int32, P(abi.Bunch)], C.c_int),
        "bmadgpu_batch_track": ([V, C.c_int32, C.c_int32], C.c_int),
        "bmadgpu_batch_set_tuning": ([V, P(BatchTuning)], C.c_int),
        "bmadgpu_batch_get_tuning": ([V, P(BatchTuning)], C.c_int),
        "bmadgpu_batch_autotune": ([V, C.c_int32, P(BatchTuning)], C.c_int),
    }
    for name, (args, res) in sig.items():
        f = getattr(lib, name, None)
        if f is None:
            continue
        f.argtypes = args
        f.restype = res
    _libs[path] = lib
    return lib


def declared_symbols(header=HEADER_PATH):
    """Function names declared in include/bmadgpu.h."""
    text = open(header).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(bmadgpu_[a-z0-9_]+)\s*\(", text)))


def check(code):
    if code != 0:
        raise BmadGpuError(code, load().bmadgpu_last_error().decode())
    return code


def check_layout():
    """Compare ctypes struct sizes with the compiled library's sizeof()."""
    lib = load()
    for i, st in enumerate((abi.Element, abi.Param, abi.Bunch, Tuning, BatchTuning, ServerConfig, JobInfo,
                            ServerStats, BunchData, LttParams, DaParams, DaPoint, Twiss, BeamInit, FmaParams, FmaPoint)):
        if lib.bmadgpu_sizeof(i) != C.sizeof(st):
            raise BmadGpuError(abi.EINVAL, "ABI size mismatch for %s" % st.__name__)


def lattice_check(elements, param):
    """Host-only validation and bookkeeping: returns (n_step per element, packed table bytes)."""
    lib = load()
    arr = abi.element_array(elements) if not isinstance(elements, C.Array) else elements
    n = len(arr)
    steps = (C.c_int32 * n)()
    nbytes = C.c_int64(0)
    check(lib.bmadgpu_lattice_check(arr, n, C.byref(param), steps, C.byref(nbytes)))
    return list(steps), nbytes.value


class Context:
    """A device context (bmadgpu_ctx): one CUDA stream plus staging buffers."""

    def __init__(self, device=0):
        lib = load()
        check_layout()
        self._h = C.c_void_p()
        check(lib.bmadgpu_ctx_create(device, C.byref(self._h)))
        d, sm, st = C.c_int32(), C.c_int32(), C.c_void_p()
        check(lib.bmadgpu_ctx_info(self._h, C.byref(d), C.byref(sm), C.byref(st)))
        self.device, self.sm_count, self.stream = d.value, sm.value, st.value

    @property
    def handle(self):
        return self._h

    def synchronize(self):
        check(load().bmadgpu_ctx_synchronize(self._h))

    def get_tuning(self):
        t = Tuning()
        check(load().bmadgpu_ctx_get_tuning(self._h, C.byref(t)))
        return dict(block=t.block, ctas_per_sm=t.ctas_per_sm, stage_smem=t.stage_smem,
                    turns_per_launch=t.turns_per_launch, compact=t.compact)

    def set_tuning(self, **kw):
        cur = self.get_tuning()
        cur.update(kw)
        t = Tuning(cur["block"], cur["ctas_per_sm"], cur["stage_smem"], cur["turns_per_launch"], cur["compact"])
        check(load().bmadgpu_ctx_set_tuning(self._h, C.byref(t)))

    @property
    def launch_count(self):
        return load().bmadgpu_ctx_launch_count(self._h)

    def measure_fp64_peak(self):
        """FP64 FLOP/s of a DFMA-chain kernel on every SM of this device."""
        f = C.c_double()
        check(load().bmadgpu_measure_fp64_peak(self._h, C.byref(f)))
        return f.value

    def adopt(self, obj):
        """Objects made on this context (batches, servers) are closed before it: their C destroy
        calls use the context's stream."""
        import weakref
        if not hasattr(self, "_children"):
            self._children = weakref.WeakSet()
        self._children.add(obj)

    def close(self):
        for obj in list(getattr(self, "_children", ())):
            obj.close()
        if self._h:
            load().bmadgpu_ctx_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Lattice:
    """Packed, device-resident element table (bmadgpu_lattice)."""

    def __init__(self, ctx, elements, param):
        lib = load()
        self.ctx = ctx
        self.elements = abi.element_array(elements) if not isinstance(elements, C.Array) else elements
        self.param = param
        self.n_ele = len(self.elements)
        self._h = C.c_void_p()
        check(lib.bmadgpu_lattice_create(ctx.handle, self.elements, self.n_ele, C.byref(param), C.byref(self._h)))

    @property
    def handle(self):
        return self._h

    def n_step(self, i):
        return load().bmadgpu_lattice_n_step(self._h, i)

    @property
    def table_bytes(self):
        return load().bmadgpu_lattice_table_bytes(self._h)

    def close(self):
        if self._h:
            load().bmadgpu_lattice_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class HostBunch:
    """Structure-of-arrays particle arrays in host memory (numpy), the bmadgpu_bunch view of a
    bunch_struct. vec is [6, n] C-contiguous so vec[i] is coordinate i of every particle."""

    def __init__(self, vec, beta, state=None, t=None, track_losses=True):
        # own copies: tracking updates these arrays in place
        self.vec = np.array(vec, dtype=np.float64, order="C", copy=True)
        n = self.vec.shape[1]
        self.beta = np.array(beta, dtype=np.float64, copy=True)
        self.state = (np.full(n, abi.ALIVE, dtype=np.int32) if state is None
                      else np.array(state, dtype=np.int32, copy=True))
        self.t = None if t is None else np.array(t, dtype=np.float64, copy=True)
        if track_losses:
            self.ix_ele = np.full(n, -1, dtype=np.int32)
            self.ix_turn = np.full(n, -1, dtype=np.int32)
            self.location = np.zeros(n, dtype=np.int32)
        else:
            self.ix_ele = self.ix_turn = self.location = None

    @classmethod
    def from_vec(cls, vec, param, **kw):
        """Particles at the upstream end with beta from pz as init_coord computes it."""
        vec = np.asarray(vec, dtype=np.float64)
        pc = param.p0c * (1 + vec[5])
        beta = np.where(vec[5] == 0, param.p0c / param.e_tot, pc / np.sqrt(pc * pc + param.mass * param.mass))
        return cls(vec, beta, **kw)

    @property
    def n(self):
        return self.vec.shape[1]

    def view(self):
        def ptr(a):
            return None if a is None else a.ctypes.data
        return abi.Bunch(self.n, ptr(self.vec), ptr(self.beta), ptr(self.t), ptr(self.state), ptr(self.ix_ele),
                         ptr(self.ix_turn), ptr(self.location))


def track_bunch(ctx, lat, bunch, n_turns=1, ix_start=0, ix_end=None, turn0=0, moments=False):
    """Track a HostBunch for n_turns over elements [ix_start, ix_end) (host buffers, copies
    included). Returns the per-turn moment sums [n_turns, 28] if moments is True."""
    lib = load()
    ix_end = lat.n_ele if ix_end is None else ix_end
    mom = np.zeros((max(n_turns, 1), abi.N_MOMENTS)) if moments else None
    v = bunch.view()
    check(lib.bmadgpu_track_bunch(ctx.handle, lat.handle, C.byref(v), ix_start, ix_end, turn0, n_turns,
                                  mom.ctypes.data if mom is not None else None))
    return mom


# ---- several GPUs: particle shards, one collective for the moments ----------------------------

def shard(n, rank, world):
    """[start, stop) of the particles rank tracks when n particles are shared by world ranks:
    contiguous ranges whose sizes differ by at most one, in rank order. Particles never interact
    on this path, so the shards are tracked independently (one process per GPU)."""
    if world < 1 or not 0 <= rank < world:
        raise BmadGpuError(abi.EINVAL, "bad rank/world")
    q, r = divmod(n, world)
    start = rank * q + min(rank, r)
    return start, start + q + (1 if rank < r else 0)


def allreduce_moments(moments, group=None):
    """The whole job's per-turn moment sums (n_live, sum vec_i, sum vec_i vec_j: [n_turns, 28]) from
    each rank's sums over its shard: one all_reduce (sum) of all reported turns at once
    (torch.distributed; NCCL for CUDA tensors, gloo for CPU ones). The reference gathers the same
    sums from its MPI workers (bsim/long_term_tracking/long_term_tracking_mpi.f90:344, 381).
    Takes a float64 torch tensor or numpy array and returns the sums as a new one of the same kind."""
    import torch
    import torch.distributed as dist
    as_numpy = isinstance(moments, np.ndarray)
    t = torch.from_numpy(np.array(moments, dtype=np.float64, copy=True)) if as_numpy else moments.clone()
    if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t.numpy() if as_numpy else t


def autotune(ctx, lat, device_bunch_view, sample_n=0):
    """Run the library's launch-shape autotuner on a device-resident bunch view (abi.Bunch of
    device pointers); returns the chosen tuning (also set on the context)."""
    t = Tuning()
    check(load().bmadgpu_autotune(ctx.handle, lat.handle, C.byref(device_bunch_view), sample_n, C.byref(t)))
    return dict(block=t.block, ctas_per_sm=t.ctas_per_sm, stage_smem=t.stage_smem,
                turns_per_launch=t.turns_per_launch, compact=t.compact)


def track1_bunch(ctx, lat, bunch, ix_ele, turn=0):
    """One element for the whole bunch: the work of track1_bunch / track1_bunch_hom."""
    v = bunch.view()
    check(load().bmadgpu_track1_bunch(ctx.handle, lat.handle, C.byref(v), ix_ele, turn))


class Batch:
    """Many lattice variants with their own particle counts, tracked together (bmadgpu_batch):
    one persistent launch per batch of turns, fed by a device work queue, replayed as a CUDA
    graph. The batch owns the device particle state; ``upload``/``download`` move a variant's
    particles (v = -1: all variants, concatenated in variant order)."""

    def __init__(self, ctx, lattices, counts):
        lib = load()
        self.ctx = ctx
        self.lattices = list(lattices)
        self.counts = [int(c) for c in counts]
        if len(self.lattices) != len(self.counts):
            raise BmadGpuError(abi.EINVAL, "one particle count per lattice")
        n = len(self.lattices)
        hl = (C.c_void_p * n)(*[l.handle.value for l in self.lattices])
        hc = (C.c_int64 * n)(*self.counts)
        self._h = C.c_void_p()
        check(lib.bmadgpu_batch_create(ctx.handle, n, hl, hc, C.byref(self._h)))
        ctx.adopt(self)
        self.offsets = np.concatenate([[0], np.cumsum(self.counts)]).astype(np.int64)

    @property
    def handle(self):
        return self._h

    @property
    def n_var(self):
        return len(self.counts)

    @property
    def total(self):
        return int(self.offsets[-1])

    def view(self, v=-1):
        """Device pointers (abi.Bunch) of variant v, or of the whole batch."""
        b = abi.Bunch()
        check(load().bmadgpu_batch_view(self._h, v, C.byref(b)))
        return b

    def upload(self, v, bunch):
        """Copy a HostBunch into variant v (v = -1: a HostBunch of all particles in batch layout).
        The copy is queued on the context stream; keep ``bunch`` alive until the next
        synchronisation (download or ctx.synchronize)."""
        hv = bunch.view()
        check(load().bmadgpu_batch_upload(self._h, v, C.byref(hv)))

    def download(self, v, bunch):
        hv = bunch.view()
        check(load().bmadgpu_batch_download(self._h, v, C.byref(hv)))

    def track(self, n_turns, turn0=0):
        """Queue n_turns turns of every variant (asynchronous; download or ctx.synchronize waits)."""
        check(load().bmadgpu_batch_track(self._h, turn0, n_turns))

    def get_tuning(self):
        t = BatchTuning()
        check(load().bmadgpu_batch_get_tuning(self._h, C.byref(t)))
        return {k: getattr(t, k) for k in _BATCH_FIELDS}

    def set_tuning(self, **kw):
        cur = self.get_tuning()
        cur.update(kw)
        t = BatchTuning(*[cur[k] for k in _BATCH_FIELDS])
        check(load().bmadgpu_batch_set_tuning(self._h, C.byref(t)))

    def autotune(self, sample_turns=0):
        t = BatchTuning()
        check(load().bmadgpu_batch_autotune(self._h, sample_turns, C.byref(t)))
        return {k: getattr(t, k) for k in _BATCH_FIELDS}

    def close(self):
        if self._h:
            load().bmadgpu_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def concat_bunches(bunches):
    """One HostBunch holding the given bunches one after another, in the batch layout
    (each bunch's [6, n] block contiguous)."""
    n = sum(b.n for b in bunches)
    out = HostBunch(np.zeros((6, n)), np.zeros(n))
    flat = out.vec.reshape(-1)
    at = 0
    for b in bunches:
        flat[6 * at:6 * (at + b.n)] = b.vec.reshape(-1)
        out.beta[at:at + b.n] = b.beta
        out.state[at:at + b.n] = b.state
        at += b.n
    out.t = np.zeros(n)
    at = 0
    for b in bunches:
        if b.t is not None:
            out.t[at:at + b.n] = b.t
        at += b.n
    return out


def split_bunch(whole, counts):
    """Inverse of concat_bunches: per-variant HostBunch copies from a batch-layout HostBunch."""
    flat = whole.vec.reshape(-1)
    out, at = [], 0
    for n in counts:
        b = HostBunch(flat[6 * at:6 * (at + n)].reshape(6, n), whole.beta[at:at + n],
                      state=whole.state[at:at + n], t=None if whole.t is None else whole.t[at:at + n])
        for f in ("ix_ele", "ix_turn", "location"):
            src = getattr(whole, f)
            if src is not None:
                setattr(b, f, np.array(src[at:at + n], copy=True))
        out.append(b)
        at += n
    return out


# ---- serving ---------------------------------------------------------------------------------

class ServerConfig(C.Structure):
    _fields_ = [("max_particles", C.c_int64), ("hbm_fraction", C.c_double), ("max_jobs", C.c_int32),
                ("element_steps", C.c_int32), ("target_live", C.c_int64), ("policy", C.c_int32),
                ("block", C.c_int32), ("ctas_per_sm", C.c_int32), ("stage_smem", C.c_int32),
                ("record_mib", C.c_int32), ("reserved", C.c_int32 * 3)]


class JobInfo(C.Structure):
    _fields_ = [("status", C.c_int32), ("rounds", C.c_int32), ("t_submit", C.c_double), ("t_admit", C.c_double),
                ("t_done", C.c_double), ("particle_turns", C.c_int64)]


class ServerStats(C.Structure):
    _fields_ = [("jobs_submitted", C.c_int64), ("jobs_done", C.c_int64), ("rounds", C.c_int64),
                ("particle_turns", C.c_int64), ("elapsed_s", C.c_double), ("latency_p50_s", C.c_double),
                ("latency_p99_s", C.c_double), ("latency_max_s", C.c_double), ("capacity", C.c_int64),
                ("peak_resident", C.c_int64), ("gpu_busy_s", C.c_double), ("gpu_idle_s", C.c_double),
                ("gpu_max_gap_s", C.c_double)]


SERVE_SRPT, SERVE_FIFO = 0, 1
JOB_QUEUED, JOB_RUNNING, JOB_DONE, JOB_CANCELLED = 0, 1, 2, 3


def _serve_sigs(lib):
    P, V = C.POINTER, C.c_void_p
    sig = {
        "bmadgpu_server_create": ([V, P(ServerConfig), P(V)], C.c_int),
        "bmadgpu_server_destroy": ([V], C.c_int),
        "bmadgpu_server_submit": ([V, V, P(abi.Bunch), C.c_int32, C.c_int32, P(C.c_int64)], C.c_int),
        "bmadgpu_server_job": ([V, C.c_int64, P(JobInfo)], C.c_int),
        "bmadgpu_server_wait": ([V, C.c_int64, C.c_double], C.c_int),
        "bmadgpu_server_get_stats": ([V, P(ServerStats)], C.c_int),
        "bmadgpu_host_alloc": ([C.c_int64, P(V)], C.c_int),
        "bmadgpu_host_free": ([V], C.c_int),
    }
    for name, (args, res) in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    return lib


class PinnedBunch(HostBunch):
    """HostBunch whose arrays live in page-locked host memory (bmadgpu_host_alloc), so the
    server's copies of it run asynchronously and overlap with tracking."""

    def __init__(self, vec, beta, state=None, t=None, track_losses=True):
        lib = _serve_sigs(load())
        vec = np.asarray(vec, dtype=np.float64)
        n = vec.shape[1]
        self._blocks = []

        def alloc(shape, dtype):
            nbytes = int(np.prod(shape)) * np.dtype(dtype).itemsize
            p = C.c_void_p()
            check(lib.bmadgpu_host_alloc(max(nbytes, 8), C.byref(p)))
            self._blocks.append(p.value)
            buf = (C.c_char * max(nbytes, 8)).from_address(p.value)
            return np.frombuffer(buf, dtype=dtype, count=int(np.prod(shape))).reshape(shape)

        self.vec = alloc((6, n), np.float64)
        self.vec[:] = vec
        self.beta = alloc((n,), np.float64)
        self.beta[:] = beta
        self.state = alloc((n,), np.int32)
        self.state[:] = abi.ALIVE if state is None else state
        self.t = None
        if t is not None:
            self.t = alloc((n,), np.float64)
            self.t[:] = t
        if track_losses:
            self.ix_ele = alloc((n,), np.int32)
            self.ix_ele[:] = -1
            self.ix_turn = alloc((n,), np.int32)
            self.ix_turn[:] = -1
            self.location = alloc((n,), np.int32)
            self.location[:] = 0
        else:
            self.ix_ele = self.ix_turn = self.location = None

    def free(self):
        lib = load()
        for p in self._blocks:
            lib.bmadgpu_host_free(p)
        self._blocks = []
        self.vec = self.beta = self.state = self.t = self.ix_ele = self.ix_turn = self.location = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Server:
    """Continuous-batching tracking server (bmadgpu_server): jobs of any lattice, particle count
    and turn count are submitted at any time and tracked together, with the particle state and the
    lattice tables resident on the device. ``submit`` returns a job id; the bunch is written back
    in place when the job is done."""

    def __init__(self, ctx, **cfg):
        lib = _serve_sigs(load())
        self.ctx = ctx
        c = ServerConfig()
        for k, v in cfg.items():
            setattr(c, k, v)
        self._h = C.c_void_p()
        check(lib.bmadgpu_server_create(ctx.handle, C.byref(c), C.byref(self._h)))
        ctx.adopt(self)
        self._keep = {}

    def submit(self, lat, bunch, n_turns, turn0=0):
        v = bunch.view()
        jid = C.c_int64()
        check(load().bmadgpu_server_submit(self._h, lat.handle, C.byref(v), turn0, n_turns, C.byref(jid)))
        self._keep[jid.value] = (lat, bunch)
        return jid.value

    def submit_fma(self, lat, bunch, n_turns, norm, orbit, tunes, fft_turns=0, z_cut=True, rf_frequency=0.0,
                   turn0=0):
        """A frequency-map job: bunch holds closed orbit + offsets; norm, orbit and tunes as
        fma_setup gives them. fma_result(jid) has the tunes once the job is done."""
        lib = load()
        lib.bmadgpu_server_submit_fma.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(abi.Bunch), C.c_int32, C.c_int32,
                                                  C.POINTER(FmaParams), C.POINTER(FmaPoint), C.POINTER(C.c_int64)]
        P = FmaParams(n_turns, fft_turns, 1 if z_cut else 0, 0, rf_frequency)
        P.norm[:] = list(np.asarray(norm, float).ravel())
        P.orbit[:] = list(np.asarray(orbit, float))
        P.tune_a, P.tune_b = tunes
        pts = (FmaPoint * max(bunch.n, 1))()
        v = bunch.view()
        jid = C.c_int64()
        check(lib.bmadgpu_server_submit_fma(self._h, lat.handle, C.byref(v), turn0, n_turns, C.byref(P), pts,
                                            C.byref(jid)))
        self._keep[jid.value] = (lat, bunch, P, pts)
        return jid.value

    def fma_result(self, jid):
        """(tunes [n, 6], status [n], turn_lost [n], ix_ele [n]) of a finished frequency-map job."""
        _, bunch, _, pts = self._keep[jid]
        n = bunch.n
        q = np.array([pts[i].tune[:] for i in range(n)]).reshape(n, 6)
        st = np.array([pts[i].status for i in range(n)], np.int32)
        tl = np.array([pts[i].turn_lost for i in range(n)], np.int32)
        ie = np.array([pts[i].ix_ele for i in range(n)], np.int32)
        return q, st, tl, ie

    def job(self, jid):
        i = JobInfo()
        check(load().bmadgpu_server_job(self._h, jid, C.byref(i)))
        return {f: getattr(i, f) for f, _ in JobInfo._fields_}

    def wait(self, jid=-1, timeout=3600.0):
        check(load().bmadgpu_server_wait(self._h, jid, timeout))

    def stats(self):
        s = ServerStats()
        check(load().bmadgpu_server_get_stats(self._h, C.byref(s)))
        return {f: getattr(s, f) for f, _ in ServerStats._fields_}

    def close(self):
        if self._h:
            load().bmadgpu_server_destroy(self._h)
            self._h = C.c_void_p()
            self._keep = {}

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---- differentiation -------------------------------------------------------------------------

def loss_grad(ctx, lat, bunch, n_turns, param_ele, checkpoint_every=16):
    """loss = mean over the bunch of x^2 + y^2 (particles alive after n_turns) and its gradient
    with respect to the strengths (k1 / k2 / k3) of the elements param_ele, by the library's
    adjoint kernel. The bunch (HostBunch) is not modified. Returns (loss, grad ndarray)."""
    lib = load()
    if not hasattr(lib, "_loss_grad_sig"):
        lib.bmadgpu_loss_grad.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(abi.Bunch), C.c_int32, C.c_int32,
                                          C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_double),
                                          C.POINTER(C.c_double)]
        lib.bmadgpu_loss_grad.restype = C.c_int
        lib._loss_grad_sig = True
    idx = np.ascontiguousarray(param_ele, dtype=np.int32)
    grad = np.zeros(len(idx))
    loss = C.c_double()
    v = bunch.view()
    check(lib.bmadgpu_loss_grad(ctx.handle, lat.handle, C.byref(v), n_turns, checkpoint_every, len(idx),
                                idx.ctypes.data_as(C.POINTER(C.c_int32)), C.byref(loss),
                                grad.ctypes.data_as(C.POINTER(C.c_double))))
    return loss.value, grad


# ---- long-term tracking outputs --------------------------------------------------------------

class BunchData(C.Structure):
    _fields_ = [("n_live", C.c_int64), ("t", C.c_double), ("sigma_t", C.c_double), ("p0c", C.c_double),
                ("centroid", C.c_double * 6), ("sigma_vec", C.c_double * 21), ("sig1", C.c_double * 6),
                ("skew", C.c_double * 3), ("kurt", C.c_double * 3), ("sigma", C.c_double * 36),
                ("emit", C.c_double * 3), ("norm_emit", C.c_double * 3), ("proj_emit", C.c_double * 3),
                ("proj_beta", C.c_double * 3), ("proj_alpha", C.c_double * 3), ("eta", C.c_double * 2),
                ("etap", C.c_double * 2), ("emit_valid", C.c_int32), ("reserved", C.c_int32)]

    def as_dict(self):
        out = {}
        for f, _ in self._fields_:
            v = getattr(self, f)
            out[f] = np.array(v[:]) if hasattr(v, "_length_") else v
        return out


class LttParams(C.Structure):
    _fields_ = [("n_turns", C.c_int32), ("averages_every_n_turns", C.c_int32), ("particle_every_n_turns", C.c_int32),
                ("output_only_last_turns", C.c_int32), ("only_live_particles_out", C.c_int32),
                ("ix_turn_start", C.c_int32), ("beam_every_n_turns", C.c_int32), ("beam_exact", C.c_int32),
                ("dead_cutoff", C.c_double), ("averages_file", C.c_char_p), ("phase_space_file", C.c_char_p),
                ("beam_file", C.c_char_p), ("core_emit_cutoff", C.c_double * 8), ("core_emit_per_mode", C.c_int32),
                ("action_angle_file", C.c_char_p), ("per_particle_file", C.c_char_p),
                ("action_angle_n_inv", C.POINTER(C.c_double))]


def _ltt_sigs(lib):
    P, V = C.POINTER, C.c_void_p
    for name, args in (("bmadgpu_bunch_stats", [V, V, P(abi.Bunch), P(BunchData)]),
                       ("bmadgpu_bunch_data_from_sums", [P(C.c_double), C.c_double, C.c_double, P(BunchData)]),
                       ("bmadgpu_ltt_run", [V, V, P(abi.Bunch), P(LttParams), P(C.c_int32)])):
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = C.c_int
    return lib


def sigma_normal_form(sigma):
    """Host-only: (emit[3], n_mat[6, 6]) of a 6x6 sigma matrix, the normal-form matrix N that
    calc_emittances_and_twiss_from_sigma_matrix returns (no GPU needed)."""
    lib = load()
    lib.bmadgpu_sigma_normal_form.argtypes = [C.POINTER(C.c_double)] * 3
    sig = np.ascontiguousarray(sigma, dtype=np.float64).reshape(36)
    emit = np.zeros(3)
    n_mat = np.zeros(36)
    check_host(lib.bmadgpu_sigma_normal_form(*(a.ctypes.data_as(C.POINTER(C.c_double)) for a in (sig, emit, n_mat))))
    return emit, n_mat.reshape(6, 6)


def bunch_data_from_sums(sums, p0c, mass):
    """Host-only: the bunch data from the 63 two-pass sums (no GPU needed)."""
    lib = _ltt_sigs(load())
    s = np.ascontiguousarray(sums, dtype=np.float64)
    bd = BunchData()
    check(lib.bmadgpu_bunch_data_from_sums(s.ctypes.data_as(C.POINTER(C.c_double)), p0c, mass, C.byref(bd)))
    return bd.as_dict()


def bunch_core_emit(ctx, lat, device_view, cutoff=0.5, combined_calc=True):
    """Core emittances (a, b, c) of a device-resident bunch as ltt_calc_bunch_data computes them
    (combined_calc: ltt%core_emit_combined_calc)."""
    lib = load()
    lib.bmadgpu_bunch_core_emit.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(abi.Bunch), C.c_double, C.c_int32,
                                            C.POINTER(C.c_double)]
    out = (C.c_double * 3)()
    check(lib.bmadgpu_bunch_core_emit(ctx.handle, lat.handle, C.byref(device_view), cutoff,
                                      1 if combined_calc else 0, out))
    return np.array(out[:])


def select_smallest(ctx, keys, n_cut):
    """Device core selection (bmadgpu_select_smallest) of the n_cut smallest of the amplitudes
    `keys` (a CUDA torch tensor of float64), ties to the lower index. Returns the mask as a numpy
    int32 array, or None where the n_cut-th smallest marks a particle that cannot be in a core."""
    import torch
    lib = load()
    lib.bmadgpu_select_smallest.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_int64, C.c_void_p,
                                            C.POINTER(C.c_int32)]
    n = keys.numel()
    mask = torch.full((n,), -7, dtype=torch.int32, device=keys.device)
    sel = C.c_int32(0)
    check(lib.bmadgpu_select_smallest(ctx.handle, keys.data_ptr(), n, n_cut, mask.data_ptr(), C.byref(sel)))
    return mask.cpu().numpy() if sel.value else None


def bunch_stats(ctx, lat, device_view):
    """Bunch data (ltt_calc_bunch_data) of a device-resident bunch."""
    lib = _ltt_sigs(load())
    bd = BunchData()
    check(lib.bmadgpu_bunch_stats(ctx.handle, lat.handle, C.byref(device_view), C.byref(bd)))
    return bd.as_dict()


def ltt_run(ctx, lat, bunch, n_turns, averages_file=None, phase_space_file=None, averages_every_n_turns=-1,
            particle_every_n_turns=-1, output_only_last_turns=0, only_live_particles_out=True, dead_cutoff=1.0,
            beam_file=None, beam_every_n_turns=-1, beam_exact=False, ix_turn_start=0, core_emit_cutoff=None,
            core_emit_combined_calc=True, action_angle_file=None, per_particle_file=None,
            action_angle_calc_uses_1turn_matrix=False):
    """long_term_tracking's beam mode for a HostBunch (updated in place); returns the turn reached.
    core_emit_cutoff: list of core fractions for the .emit file (None: the reference's [0.5];
    []: no core columns); core_emit_combined_calc False: a core per normal mode.
    action_angle_file / per_particle_file: the reference's action-angle and per-particle outputs;
    action_angle_calc_uses_1turn_matrix: actions from make_N of the one-turn matrix about the
    closed orbit (RF on), as the reference's option does, instead of the bunch's normal form."""
    lib = _ltt_sigs(load())
    p = LttParams(n_turns, averages_every_n_turns, particle_every_n_turns, output_only_last_turns,
                  1 if only_live_particles_out else 0, ix_turn_start, beam_every_n_turns, 1 if beam_exact else 0,
                  dead_cutoff, averages_file.encode() if averages_file else None,
                  phase_space_file.encode() if phase_space_file else None,
                  beam_file.encode() if beam_file else None)
    if core_emit_cutoff is not None:
        cuts = list(core_emit_cutoff)[:8]
        p.core_emit_cutoff[:] = cuts + [-1.0] * (8 - len(cuts))
    p.core_emit_per_mode = 0 if core_emit_combined_calc else 1
    p.action_angle_file = action_angle_file.encode() if action_angle_file else None
    p.per_particle_file = per_particle_file.encode() if per_particle_file else None
    n_inv = None
    if action_angle_file and action_angle_calc_uses_1turn_matrix:
        orbit = closed_orbit(ctx, lat)[0]
        t6 = one_turn_matrix(ctx, lat, orbit, rf_on=True)[0]
        if np.all(t6[0:5, 5] == 0):
            raise BmadGpuError(abi.EINVAL, "action_angle_calc_uses_1turn_matrix needs the RF on")
        n_inv = np.ascontiguousarray(np.linalg.inv(make_n(t6)).ravel())
        p.action_angle_n_inv = n_inv.ctypes.data_as(C.POINTER(C.c_double))
    done = C.c_int32()
    v = bunch.view()
    check(lib.bmadgpu_ltt_run(ctx.handle, lat.handle, C.byref(v), C.byref(p), C.byref(done)))
    return done.value


BEAM_ALIVE_ONLY, BEAM_APPEND, BEAM_EXACT, BEAM_AT_ELEMENT = 1, 2, 4, 8


def beam_write(path, bunch, param, s_position=0.0, flags=0):
    """Bmad ASCII (version 4) beam file of a HostBunch."""
    lib = load()
    lib.bmadgpu_beam_write_ascii.argtypes = [C.c_char_p, C.POINTER(abi.Bunch), C.POINTER(abi.Param), C.c_double,
                                             C.c_int32]
    v = bunch.view()
    check_host(lib.bmadgpu_beam_write_ascii(path.encode(), C.byref(v), C.byref(param), s_position, flags))


def beam_read(path, param):
    """HostBunch from a Bmad ASCII beam file (version 4, or the older ASCII::3 layout)."""
    lib = load()
    lib.bmadgpu_beam_read_ascii.argtypes = [C.c_char_p, C.POINTER(abi.Param), C.POINTER(abi.Bunch),
                                            C.POINTER(C.c_int64)]
    n = C.c_int64()
    check_host(lib.bmadgpu_beam_read_ascii(path.encode(), C.byref(param), None, C.byref(n)))
    b = HostBunch(np.zeros((6, n.value)), np.zeros(n.value), t=np.zeros(n.value))
    v = b.view()
    check_host(lib.bmadgpu_beam_read_ascii(path.encode(), C.byref(param), C.byref(v), C.byref(n)))
    return b


def beam_write_hdf5(path, bunch, param, s_position=0.0, flags=0):
    """Bmad openPMD beam file (HDF5) of a HostBunch, or of a list of them (one bunch group each), as
    hdf5_write_beam lays it out."""
    lib = load()
    if isinstance(bunch, (list, tuple)):
        lib.bmadgpu_beam_write_hdf5_bunches.argtypes = [C.c_char_p, C.POINTER(abi.Bunch), C.c_int32,
                                                        C.POINTER(abi.Param), C.c_double, C.c_int32]
        views = (abi.Bunch * len(bunch))(*[b.view() for b in bunch])
        check_host(lib.bmadgpu_beam_write_hdf5_bunches(path.encode(), views, len(bunch), C.byref(param), s_position,
                                                       flags))
        return
    lib.bmadgpu_beam_write_hdf5.argtypes = [C.c_char_p, C.POINTER(abi.Bunch), C.POINTER(abi.Param), C.c_double,
                                            C.c_int32]
    v = bunch.view()
    check_host(lib.bmadgpu_beam_write_hdf5(path.encode(), C.byref(v), C.byref(param), s_position, flags))


def beam_read_hdf5(path, param, ix_bunch=0, flags=0):
    """(HostBunch of bunch ix_bunch, number of bunches) from a Bmad openPMD beam file, as
    hdf5_read_beam reads it without an element (flags BEAM_AT_ELEMENT: with the beginning element)."""
    lib = load()
    lib.bmadgpu_beam_read_hdf5.argtypes = [C.c_char_p, C.POINTER(abi.Param), C.c_int32, C.c_int32,
                                           C.POINTER(abi.Bunch), C.POINTER(C.c_int64), C.POINTER(C.c_int32)]
    n, nb = C.c_int64(), C.c_int32()
    check_host(lib.bmadgpu_beam_read_hdf5(path.encode(), C.byref(param), ix_bunch, flags, None, C.byref(n),
                                          C.byref(nb)))
    b = HostBunch(np.zeros((6, n.value)), np.zeros(n.value), t=np.zeros(n.value))
    v = b.view()
    check_host(lib.bmadgpu_beam_read_hdf5(path.encode(), C.byref(param), ix_bunch, flags, C.byref(v), C.byref(n),
                                          C.byref(nb)))
    return b, nb.value


def write_beam_file(path, bunch, param, s_position=0.0, flags=0):
    """write_beam_file: HDF5 for names ending in .h5 or .hdf5, else Bmad's ASCII layout."""
    lib = load()
    lib.bmadgpu_beam_write_file.argtypes = [C.c_char_p, C.POINTER(abi.Bunch), C.POINTER(abi.Param), C.c_double,
                                            C.c_int32]
    v = bunch.view()
    check_host(lib.bmadgpu_beam_write_file(path.encode(), C.byref(v), C.byref(param), s_position, flags))


def read_beam_file(path, param):
    """read_beam_file: a HostBunch (the first bunch of an HDF5 file) in the format the name gives."""
    lib = load()
    lib.bmadgpu_beam_read_file.argtypes = [C.c_char_p, C.POINTER(abi.Param), C.POINTER(abi.Bunch),
                                           C.POINTER(C.c_int64)]
    n = C.c_int64()
    check_host(lib.bmadgpu_beam_read_file(path.encode(), C.byref(param), None, C.byref(n)))
    b = HostBunch(np.zeros((6, n.value)), np.zeros(n.value), t=np.zeros(n.value))
    v = b.view()
    check_host(lib.bmadgpu_beam_read_file(path.encode(), C.byref(param), C.byref(v), C.byref(n)))
    return b


def check_host(code):
    """Status check for the host-only calls (they set no last-error message)."""
    if code != 0:
        raise BmadGpuError(code, "host call failed")


# ---- dynamic aperture ------------------------------------------------------------------------

class DaParams(C.Structure):
    _fields_ = [("x_init", C.c_double), ("y_init", C.c_double), ("abs_accuracy", C.c_double),
                ("rel_accuracy", C.c_double), ("n_turn", C.c_int32), ("max_iterations", C.c_int32)]


class DaPoint(C.Structure):
    _fields_ = [("x", C.c_double), ("y", C.c_double), ("i_turn", C.c_int32), ("ix_ele", C.c_int32),
                ("plane", C.c_int32), ("iterations", C.c_int32)]


def da_scan(ctx, lat, theta, n_turn, x_init=1e-3, y_init=1e-3, abs_accuracy=1e-5, rel_accuracy=0.0, orb0=None,
            max_iterations=0):
    """Dynamic-aperture points along rays theta (dynamic_aperture_point for all rays at once).
    Returns a list of dicts (x, y, i_turn, ix_ele, plane, iterations)."""
    lib = load()
    lib.bmadgpu_da_scan.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.POINTER(C.c_double),
                                    C.POINTER(C.c_double), C.POINTER(DaParams), C.POINTER(DaPoint)]
    th = np.ascontiguousarray(theta, dtype=np.float64)
    n = len(th)
    o = None if orb0 is None else np.ascontiguousarray(orb0, dtype=np.float64).reshape(n, 6)
    pts = (DaPoint * max(n, 1))()
    prm = DaParams(x_init, y_init, abs_accuracy, rel_accuracy, n_turn, max_iterations)
    check(lib.bmadgpu_da_scan(ctx.handle, lat.handle, n, th.ctypes.data_as(C.POINTER(C.c_double)),
                              None if o is None else o.ctypes.data_as(C.POINTER(C.c_double)), C.byref(prm), pts))
    return [{f: getattr(pts[i], f) for f, _ in DaPoint._fields_} for i in range(n)]


# ---- optics: closed orbit, one-turn matrix, periodic Twiss, matched beam ---------------------

TWISS_OK, TWISS_IN_STOP_BAND, TWISS_NON_SYMPLECTIC, TWISS_UNSTABLE, TWISS_UNSTABLE_A, TWISS_UNSTABLE_B = 1, 2, 3, 4, 5, 6


class Twiss(C.Structure):
    _fields_ = ([(n, C.c_double) for n in (
        "beta_a alpha_a gamma_a phi_a beta_b alpha_b gamma_b phi_b "
        "eta_a etap_a deta_ds_a eta_b etap_b deta_ds_b eta_x etap_x deta_ds_x eta_y etap_y deta_ds_y").split()]
        + [("c_mat", C.c_double * 4), ("gamma_c", C.c_double), ("growth_rate", C.c_double),
           ("symp_error", C.c_double), ("status", C.c_int32), ("reserved", C.c_int32)])

    def as_dict(self):
        d = {f: getattr(self, f) for f, _ in self._fields_ if f not in ("c_mat", "reserved")}
        d["c_mat"] = np.array(self.c_mat[:]).reshape(2, 2)
        return d


class BeamInit(C.Structure):
    _fields_ = ([(n, C.c_double) for n in "a_emit b_emit sig_z sig_pz dpz_dz sig_z_jitter sig_pz_jitter".split()]
                + [("center", C.c_double * 6), ("center_jitter", C.c_double * 6), ("sigma_cutoff", C.c_double),
                   ("seed", C.c_uint64), ("renorm_center", C.c_int32), ("renorm_sigma", C.c_int32)])


def _dptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def one_turn_matrix(ctx, lat, orbit, rf_on=True):
    """(mat[6, 6], orbit after one turn) about `orbit` by central differences of device tracking."""
    lib = load()
    lib.bmadgpu_one_turn_matrix.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(C.c_double), C.c_int32,
                                            C.POINTER(C.c_double), C.POINTER(C.c_double)]
    o = np.ascontiguousarray(orbit, dtype=np.float64).copy()
    end, mat = np.zeros(6), np.zeros(36)
    check(lib.bmadgpu_one_turn_matrix(ctx.handle, lat.handle, _dptr(o), 1 if rf_on else 0, _dptr(end), _dptr(mat)))
    return mat.reshape(6, 6), end


def closed_orbit(ctx, lat, dim=0, guess=None, rel_tol=0.0, abs_tol=0.0, max_iter=0):
    """closed_orbit_calc at the lattice start: (orbit[6], one-turn matrix[6, 6], iterations)."""
    lib = load()
    lib.bmadgpu_closed_orbit.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.POINTER(C.c_double),
                                         C.POINTER(C.c_double), C.c_double, C.c_double, C.c_int32,
                                         C.POINTER(C.c_int32)]
    o = np.zeros(6) if guess is None else np.ascontiguousarray(guess, dtype=np.float64).copy()
    mat = np.zeros(36)
    it = C.c_int32()
    check(lib.bmadgpu_closed_orbit(ctx.handle, lat.handle, dim, _dptr(o), _dptr(mat), rel_tol, abs_tol, max_iter,
                                   C.byref(it)))
    return o, mat.reshape(6, 6), it.value


def twiss_from_mat6(mat, orb0=None):
    """Periodic Twiss of a one-turn matrix (host-only); a dict of the bmadgpu_twiss fields."""
    lib = load()
    lib.bmadgpu_twiss_from_mat6.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(Twiss)]
    m = np.ascontiguousarray(mat, dtype=np.float64).reshape(36)
    o = None if orb0 is None else np.ascontiguousarray(orb0, dtype=np.float64)
    tw = Twiss()
    check_host(lib.bmadgpu_twiss_from_mat6(_dptr(m), None if o is None else _dptr(o), C.byref(tw)))
    return tw.as_dict()


def philox4x32_10(counter, key):
    """The Philox4x32-10 block function of the beam generator (host-only)."""
    lib = load()
    ctr = (C.c_uint32 * 4)(*counter)
    k = (C.c_uint32 * 2)(*key)
    out = (C.c_uint32 * 4)()
    check_host(lib.bmadgpu_philox4x32_10(ctr, k, out))
    return [int(v) for v in out]


def gaussian_deviates(ctx, seed, n, sigma_cutoff=0.0):
    """The deviates the beam generator draws for (seed, sigma_cutoff, n): array [6 * n + 8]."""
    import torch
    lib = load()
    lib.bmadgpu_gaussian_deviates.argtypes = [C.c_void_p, C.c_uint64, C.c_double, C.c_int64, C.c_void_p]
    d = torch.empty(6 * n + 8, dtype=torch.float64, device="cuda:%d" % ctx.device)
    check(lib.bmadgpu_gaussian_deviates(ctx.handle, seed, sigma_cutoff, n, d.data_ptr()))
    return d.cpu().numpy()


def beam_init_gaussian(ctx, param, twiss, n, seed=0, a_emit=1e-9, b_emit=10e-12, sig_z=3e-3, sig_pz=1e-3,
                       dpz_dz=0.0, sig_z_jitter=0.0, sig_pz_jitter=0.0, center=None, center_jitter=None,
                       sigma_cutoff=0.0, renorm_center=True, renorm_sigma=True, normals=None, orbit=None):
    """Matched Gaussian bunch of n particles generated on the device (init_bunch_distribution with
    RAN_GAUSS); returns a HostBunch (vec, beta, t, state). twiss: a Twiss or its dict."""
    import torch
    lib = load()
    lib.bmadgpu_beam_init_gaussian.argtypes = [C.c_void_p, C.POINTER(abi.Param), C.POINTER(Twiss),
                                               C.POINTER(BeamInit), C.c_void_p, C.POINTER(C.c_double),
                                               C.POINTER(abi.Bunch)]
    if isinstance(twiss, dict):
        tw = Twiss()
        for f, _ in Twiss._fields_:
            if f == "c_mat":
                tw.c_mat[:] = list(np.asarray(twiss["c_mat"], float).ravel())
            elif f in twiss:
                setattr(tw, f, twiss[f])
    else:
        tw = twiss
    bi = BeamInit(a_emit, b_emit, sig_z, sig_pz, dpz_dz, sig_z_jitter, sig_pz_jitter)
    bi.center[:] = list(center) if center is not None else [0.0] * 6
    bi.center_jitter[:] = list(center_jitter) if center_jitter is not None else [0.0] * 6
    bi.sigma_cutoff, bi.seed = sigma_cutoff, seed
    bi.renorm_center, bi.renorm_sigma = int(bool(renorm_center)), int(bool(renorm_sigma))
    dev = "cuda:%d" % ctx.device
    vec = torch.empty(6 * n, dtype=torch.float64, device=dev)
    beta = torch.empty(n, dtype=torch.float64, device=dev)
    t = torch.empty(n, dtype=torch.float64, device=dev)
    state = torch.empty(n, dtype=torch.int32, device=dev)
    nd = None
    if normals is not None:
        nd = torch.from_numpy(np.ascontiguousarray(normals, dtype=np.float64)).to(dev)
        assert nd.numel() == 6 * n + 8
    o = None if orbit is None else np.ascontiguousarray(orbit, dtype=np.float64)
    view = abi.Bunch(n, vec.data_ptr(), beta.data_ptr(), t.data_ptr(), state.data_ptr(), None, None, None)
    check(lib.bmadgpu_beam_init_gaussian(ctx.handle, C.byref(param), C.byref(tw), C.byref(bi),
                                         None if nd is None else nd.data_ptr(), None if o is None else _dptr(o),
                                         C.byref(view)))
    return HostBunch(vec.cpu().numpy().reshape(6, n), beta.cpu().numpy(), state=state.cpu().numpy(),
                     t=t.cpu().numpy())


# ---- frequency-map analysis ------------------------------------------------------------------

class FmaParams(C.Structure):
    _fields_ = [("n_turn", C.c_int32), ("fft_turns", C.c_int32), ("z_cut", C.c_int32), ("reserved", C.c_int32),
                ("rf_frequency", C.c_double), ("norm", C.c_double * 36), ("orbit", C.c_double * 6),
                ("tune_a", C.c_double), ("tune_b", C.c_double)]


class FmaPoint(C.Structure):
    _fields_ = [("tune", C.c_double * 6), ("status", C.c_int32), ("turn_lost", C.c_int32), ("ix_ele", C.c_int32),
                ("reserved", C.c_int32)]


def mat_eigen(mat):
    """Eigenvalues and eigenvectors (rows) of a one-turn matrix paired and ordered by plane as
    mat_eigen does (sim_utils/matrix/mat_eigen.f90:37-187) for stable modes: LAPACK geev, pairs
    assigned to the plane they live in, the odd member of each pair the one of positive
    symplectic norm, phase normalised."""
    m = np.asarray(mat, float)
    n = m.shape[0]
    nn = n // 2
    w, vr = np.linalg.eig(m)
    if np.any(w.imag == 0):
        raise BmadGpuError(abi.EINVAL, "unstable mode: no complex eigenvalue pair")
    pos = [p for p in range(n) if w[p].imag > 0]
    amp = np.zeros((nn, nn))
    for ii, p in enumerate(pos):
        re, im = vr[:, p].real, vr[:, p].imag
        for kk in range(nn):
            amp[kk, ii] = np.sum(re[2 * kk:2 * kk + 2] ** 2) + np.sum(im[2 * kk:2 * kk + 2] ** 2)
        amp[:, ii] /= np.sum(amp[:, ii])
    sort = np.zeros(nn, int)
    for _ in range(nn):
        amp2 = amp.copy()
        dmax = np.zeros(nn)
        for j in range(nn):
            mx = int(np.argmax(amp2[j]))
            amp2[j, mx] = -1
            dmax[j] = amp[j, mx] - amp[j, int(np.argmax(amp2[j]))]
        k = int(np.argmax(dmax))
        mx = int(np.argmax(amp[k]))
        sort[mx] = k
        amp[k, :] = 0
        amp[:, mx] = 0
    vals = np.zeros(n, complex)
    vecs = np.zeros((n, n), complex)
    for ii, p in enumerate(pos):
        j = 2 * sort[ii]
        e1, e2 = np.conj(vr[:, p]), vr[:, p]
        l1, l2 = np.conj(w[p]), w[p]
        fnorm = sum(2 * np.imag(np.conj(e1[jj]) * e1[jj + 1]) for jj in range(0, n, 2))
        if fnorm < 0:
            e1, e2, l1, l2, fnorm = e2, e1, l2, l1, -fnorm
        sgn = 1 / math.sqrt(fnorm) if abs(e1[j]) == 0 else abs(e1[j]) / (math.sqrt(fnorm) * e1[j])
        vals[j], vals[j + 1] = l1, l2
        vecs[j], vecs[j + 1] = sgn * e1, np.conj(sgn) * e2
    return vals, vecs


def make_n(t6):
    """N of make_N (bmad/modules/mode3_mod.f90:825-912) for a one-turn matrix with three stable
    modes, ordered by plane dominance: eigen_decomp_6mat (:449-529; LAPACK geev through
    numpy.linalg.eig, evec(:, 2k-1) = VR(2k-1) + i VR(2k) and its conjugate, each pair conjugated
    if Im(evec^T S evec)(2k-1, 2k) < 0), order_evecs_by_plane_dominance (:661-687),
    normalize_evecs (:1129-1154), N = Re(evec) Qr - Im(evec) Qi with m = 1/sqrt(2), and the
    rotations that make N(1,2), N(3,4), N(5,6) zero (MyTan, :533-544)."""
    m6 = np.asarray(t6, float)
    w, v = np.linalg.eig(m6)
    S = np.zeros((6, 6))
    for k in range(3):
        S[2 * k, 2 * k + 1], S[2 * k + 1, 2 * k] = 1.0, -1.0
    evec = np.zeros((6, 6), complex)
    ev = np.zeros(6, complex)
    for k in (0, 2, 4):
        if w[k].imag <= 0:
            raise BmadGpuError(abi.EINVAL, "make_N: the one-turn matrix has an unstable mode")
        evec[:, k], evec[:, k + 1] = v[:, k], np.conj(v[:, k])
        ev[k], ev[k + 1] = w[k], np.conj(w[k])
    check_mat = evec.T @ S @ evec
    for k in (0, 2, 4):
        if check_mat[k, k + 1].imag < 0:
            evec[:, k:k + 2] = np.conj(evec[:, k:k + 2])
            ev[k:k + 2] = np.conj(ev[k:k + 2])
    pair1 = int(np.argmax(np.abs(evec[0, [0, 2, 4]].real)))
    vec = np.abs(evec[2, [0, 2, 4]].real)
    vec[pair1] = -1
    pair2 = int(np.argmax(vec))
    pair3 = 3 - pair1 - pair2
    idx = [2 * pair1, 2 * pair1 + 1, 2 * pair2, 2 * pair2 + 1, 2 * pair3, 2 * pair3 + 1]
    evec = evec[:, idx]
    mat = np.conj(evec).T @ S @ evec
    norms = [math.sqrt(abs(mat[k, k])) for k in (0, 2, 4)]
    if min(norms) == 0:
        raise BmadGpuError(abi.EINVAL, "make_N: cannot normalise the eigenvectors (is the RF off?)")
    for j, k in enumerate((0, 2, 4)):
        evec[:, k:k + 2] = evec[:, k:k + 2] / norms[j]
    mq = 1.0 / math.sqrt(2.0)
    Qr, Qi = np.zeros((6, 6)), np.zeros((6, 6))
    for k in (0, 2, 4):
        Qr[k, k] = Qr[k + 1, k] = mq
        Qi[k, k + 1], Qi[k + 1, k + 1] = mq, -mq
    N = evec.real @ Qr - evec.imag @ Qi

    def my_tan(y, x):
        a = math.atan2(y, x)
        return a if y >= 0 else a + 2.0 * math.pi

    R = np.zeros((6, 6))
    for k in (0, 2, 4):
        th = my_tan(N[k, k + 1], N[k, k])
        c, s_ = math.cos(th), math.sin(th)
        R[k:k + 2, k:k + 2] = [[c, -s_], [s_, c]]
    return N @ R


def fma_normalization(mat6):
    """The matrix frequency_map applies to (vec - co) each turn (frequency_map.f90:200-212): with
    mat6(6,5) == 0 the inverse of the decoupling V on (x, px, y, py); otherwise the inverse of T,
    whose rows are the real and minus imaginary parts of the ordered eigenvectors (as psv Tinv)."""
    m = np.asarray(mat6, float)
    if m[5, 4] == 0:
        tw = twiss_from_mat6(m)
        Cm, g = tw["c_mat"], tw["gamma_c"]
        Vinv = np.eye(6)
        Vinv[:2, :2] = Vinv[2:4, 2:4] = g * np.eye(2)
        Vinv[:2, 2:4] = -Cm
        Vinv[2:4, :2] = np.array([[Cm[1, 1], -Cm[0, 1]], [-Cm[1, 0], Cm[0, 0]]])
        return Vinv
    _, vecs = mat_eigen(m)
    T = np.zeros((6, 6))
    for i in range(0, 6, 2):
        T[i] = vecs[i].real
        T[i + 1] = -vecs[i].imag
    return np.linalg.inv(T).T


def fma_setup(ctx, lat):
    """(closed orbit, normalisation, ring tunes) as frequency_map computes them before its grid
    loop (twiss_and_track with the RF on, frequency_map.f90:128-212)."""
    orbit = closed_orbit(ctx, lat)[0]
    norm = fma_normalization(one_turn_matrix(ctx, lat, orbit, rf_on=True)[0])
    tw = twiss_from_mat6(one_turn_matrix(ctx, lat, orbit, rf_on=False)[0], orbit)
    return orbit, norm, (tw["phi_a"] / (2 * math.pi), tw["phi_b"] / (2 * math.pi))


def fma(ctx, lat, offsets, n_turn, fft_turns=0, z_cut=True, rf_frequency=0.0, orbit=None, norm=None, tunes=None):
    """frequency_map for particles at closed orbit + offsets[n, 6]. The closed orbit, the
    normalisation and the ring tunes default to what the reference computes (fma_setup).
    Returns (tunes[n, 6], status[n], turn_lost[n], ix_ele[n])."""
    lib = load()
    lib.bmadgpu_fma.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.POINTER(C.c_double), C.POINTER(FmaParams),
                                C.POINTER(FmaPoint)]
    off = np.ascontiguousarray(offsets, dtype=np.float64).reshape(-1, 6)
    n = off.shape[0]
    if orbit is None or norm is None or tunes is None:
        o, nm, tn = fma_setup(ctx, lat)
        orbit = o if orbit is None else orbit
        norm = nm if norm is None else norm
        tunes = tn if tunes is None else tunes
    P = FmaParams(n_turn, fft_turns, 1 if z_cut else 0, 0, rf_frequency)
    P.norm[:] = list(np.asarray(norm, float).ravel())
    P.orbit[:] = list(np.asarray(orbit, float))
    P.tune_a, P.tune_b = tunes
    pts = (FmaPoint * max(n, 1))()
    check(lib.bmadgpu_fma(ctx.handle, lat.handle, n, _dptr(off), C.byref(P), pts))
    q = np.array([pts[i].tune[:] for i in range(n)]).reshape(n, 6)
    st = np.array([pts[i].status for i in range(n)], np.int32)
    tl = np.array([pts[i].turn_lost for i in range(n)], np.int32)
    ie = np.array([pts[i].ix_ele for i in range(n)], np.int32)
    return q, st, tl, ie


def fma_write(path, offsets, tunes, status, append=False):
    """The reference's .fm table (host-only)."""
    lib = load()
    lib.bmadgpu_fma_write.argtypes = [C.c_char_p, C.c_int32, C.POINTER(C.c_double), C.POINTER(FmaPoint), C.c_int32]
    off = np.ascontiguousarray(offsets, dtype=np.float64).reshape(-1, 6)
    n = off.shape[0]
    pts = (FmaPoint * max(n, 1))()
    for i in range(n):
        pts[i].tune[:] = list(np.asarray(tunes[i], float))
        pts[i].status = int(status[i])
    check_host(lib.bmadgpu_fma_write(path.encode(), n, _dptr(off), pts, 1 if append else 0))


def naff(ctx, signals, n_comp, zero_first=False):
    """NAFF of complex signals [n_signals, n_samples] on the device: (freqs [n, n_comp],
    amps [n, n_comp] complex) as naff_mod's naff returns them."""
    lib = load()
    lib.bmadgpu_naff.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.POINTER(C.c_double), C.c_int32, C.c_int32,
                                 C.POINTER(C.c_double), C.POINTER(C.c_double)]
    sig = np.atleast_2d(np.asarray(signals, dtype=np.complex128))
    n, m = sig.shape
    data = np.ascontiguousarray(sig).view(np.float64)
    freqs = np.zeros((n, n_comp))
    amps = np.zeros((n, n_comp), np.complex128)
    check(lib.bmadgpu_naff(ctx.handle, n, m, _dptr(data), n_comp, 1 if zero_first else 0, _dptr(freqs),
                           amps.view(np.float64).ctypes.data_as(C.POINTER(C.c_double))))
    return freqs, amps


def selftest_division(ctx, n=1 << 30, seed=1):
    """Mismatching pairs of the maps' shared-reciprocal division against a / b on the device
    (bmadgpu_selftest_division); 0 is the only correct answer."""
    lib = load()
    lib.bmadgpu_selftest_division.argtypes = [C.c_void_p, C.c_int64, C.c_uint64, C.POINTER(C.c_int64)]
    m = C.c_int64()
    check(lib.bmadgpu_selftest_division(ctx.handle, n, seed, C.byref(m)))
    return m.value
