"""Python handle on the engine's C ABI (include/cqg.h, include/cqg_model.h).

This is thin plumbing for tests and benchmarks; the engine itself is the shared
library ``_lib/libcqg.so`` (host C++ + sm_100a CUDA).  There is no fallback: if the
library is missing or no CUDA device is present, the GPU entry points raise.
"""
import ctypes as C
import os

import numpy as np

from . import _abi as A

_HERE = os.path.dirname(os.path.abspath(__file__))
# the in-tree build; CQG_LIBRARY selects another build of the same library
LIB_PATH = os.environ.get("CQG_LIBRARY") or os.path.join(_HERE, "_lib", "libcqg.so")
_lib = None


class EngineError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("cqg error %d: %s" % (code, msg))
        self.code = code


def lib():
    """Loads libcqg.so (built by cppqed_b200.build)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise EngineError(A.CQG_E_NODEVICE, "engine library not built: " + LIB_PATH)
        _lib = A.bind(C.CDLL(LIB_PATH), A.ENGINE_PROTOTYPES)
    return _lib


def check(rc):
    if rc != A.CQG_OK:
        raise EngineError(rc, lib().cqg_last_error().decode())
    return rc


def device_count():
    n = C.c_int(0)
    rc = lib().cqg_device_count(C.byref(n))
    return n.value if rc == A.CQG_OK else 0


def to_c(psi):
    psi = np.ascontiguousarray(psi, dtype=np.complex128)
    return psi.ctypes.data_as(C.POINTER(A.cqg_complex)), psi


class Model:
    """A workload built from a reference-style script command line (cqg_model_create)."""

    def __init__(self, script, args=()):
        args = [str(a) for a in args]
        argv = (C.c_char_p * max(len(args), 1))(*[a.encode() for a in args])
        h = C.c_void_p()
        check(lib().cqg_model_create(script.encode(), len(args), argv, C.byref(h)))
        self._h = h
        self.script = script
        self.args = args

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.cqg_model_destroy(self._h)
            self._h = None

    @property
    def desc(self):
        d = C.POINTER(A.cqg_system_desc)()
        check(lib().cqg_model_desc(self._h, C.byref(d)))
        return d

    @property
    def dim(self):
        n = C.c_int64()
        check(lib().cqg_model_dimension(self._h, C.byref(n)))
        return n.value

    @property
    def n_avr(self):
        n = C.c_int32()
        check(lib().cqg_model_n_avr(self._h, C.byref(n)))
        return n.value

    def initial_state(self):
        psi = np.zeros(self.dim, dtype=np.complex128)
        check(lib().cqg_model_initial_state(self._h, psi.ctypes.data_as(C.POINTER(A.cqg_complex))))
        return psi

    def run_pars(self):
        rp = A.cqg_run_pars()
        check(lib().cqg_model_run_pars(self._h, C.byref(rp)))
        return rp

    def process(self, avr):
        a = np.array(avr, dtype=np.float64, copy=True)
        check(lib().cqg_model_process(self._h, a.ctypes.data_as(C.POINTER(C.c_double))))
        return a

    def key(self):
        buf = C.create_string_buffer(8192)
        check(lib().cqg_model_key(self._h, buf, 8192))
        return [s for s in buf.value.decode().split("\n") if s]


class System:
    """Device-resident lowered system (cqg_system_create)."""

    def __init__(self, desc):
        h = C.c_void_p()
        check(lib().cqg_system_create(desc, C.byref(h)))
        self._h = h

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.cqg_system_destroy(self._h)
            self._h = None


def mcwf_pars(**kw):
    p = A.cqg_mcwf_pars()
    lib().cqg_mcwf_pars_default(C.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


class Ensemble:
    """An ensemble of MCWF trajectories on the device (cqg_ensemble_create / cqg_batch_create)."""

    def __init__(self, system, psi0, n_traj, pars):
        self._keep = [system]
        h = C.c_void_p()
        p, arr = to_c(psi0)
        check(lib().cqg_ensemble_create(system._h, p, int(n_traj), C.byref(pars), C.byref(h)))
        self._h = h
        self.n_traj = int(n_traj)
        self._init_sizes()

    @classmethod
    def batch(cls, systems, sys_index, psi0s, pars):
        """Trajectories over several systems; psi0s is a list of initial states (one per trajectory)."""
        self = cls.__new__(cls)
        self._keep = list(systems)
        arr = (C.c_void_p * len(systems))(*[s._h.value for s in systems])
        idx = np.ascontiguousarray(sys_index, dtype=np.int32)
        offs = np.zeros(len(psi0s), dtype=np.int64)
        flat = []
        o = 0
        for i, p in enumerate(psi0s):
            offs[i] = o
            o += len(p)
            flat.append(np.asarray(p, dtype=np.complex128))
        flat = np.ascontiguousarray(np.concatenate(flat))
        h = C.c_void_p()
        check(lib().cqg_batch_create(C.cast(arr, C.POINTER(C.c_void_p)), len(systems),
                                     idx.ctypes.data_as(C.POINTER(C.c_int32)),
                                     flat.ctypes.data_as(C.POINTER(A.cqg_complex)),
                                     offs.ctypes.data_as(C.POINTER(C.c_int64)), len(psi0s), C.byref(pars),
                                     C.byref(h)))
        self._h = h
        self.n_traj = len(psi0s)
        self._init_sizes()
        return self

    def _init_sizes(self):
        n = C.c_int64()
        a = C.c_int32()
        check(lib().cqg_ensemble_size(self._h, C.byref(n), C.byref(a)))
        self.n_avr = a.value

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.cqg_ensemble_destroy(self._h)
            self._h = None

    def _avr_buf(self, n):
        return np.zeros((n, self.n_avr + 1), dtype=np.float64)

    def run(self, Dt, n_intervals):
        """Advances every trajectory n_intervals times by Dt.  Returns the ensemble sums after
        each interval, shape (n_intervals, n_avr + 1): the linear averages, then dtDid."""
        out = self._avr_buf(n_intervals)
        check(lib().cqg_ensemble_run(self._h, float(Dt), int(n_intervals),
                                     out.ctypes.data_as(C.POINTER(C.c_double))))
        return out

    def advance_to(self, t_end):
        out = self._avr_buf(1)
        check(lib().cqg_ensemble_advance_to(self._h, float(t_end), out.ctypes.data_as(C.POINTER(C.c_double))))
        return out[0]

    def steps(self, n_steps, T):
        """n_steps MCWF steps of size T - t per trajectory (0: averages only); sums as in run."""
        out = self._avr_buf(1)
        check(lib().cqg_ensemble_steps(self._h, int(n_steps), float(T), out.ctypes.data_as(C.POINTER(C.c_double))))
        return out[0]

    def traj_averages(self):
        out = np.zeros((self.n_traj, self.n_avr + 1), dtype=np.float64)
        check(lib().cqg_ensemble_traj_averages(self._h, out.ctypes.data_as(C.POINTER(C.c_double))))
        return out

    def state(self, i, dim):
        psi = np.zeros(dim, dtype=np.complex128)
        check(lib().cqg_ensemble_get_state(self._h, int(i), psi.ctypes.data_as(C.POINTER(A.cqg_complex))))
        return psi

    def set_state(self, i, psi):
        p, arr = to_c(psi)
        check(lib().cqg_ensemble_set_state(self._h, int(i), p))

    def times(self):
        t = np.zeros(self.n_traj)
        did = np.zeros(self.n_traj)
        tr = np.zeros(self.n_traj)
        P = C.POINTER(C.c_double)
        check(lib().cqg_ensemble_get_times(self._h, t.ctypes.data_as(P), did.ctypes.data_as(P), tr.ctypes.data_as(P)))
        return t, did, tr

    def counters(self):
        c = np.zeros((self.n_traj, 8), dtype=np.uint64)
        check(lib().cqg_ensemble_get_counters(self._h, c.ctypes.data_as(C.POINTER(C.c_uint64))))
        return c

    def logger_maxima(self):
        """Per trajectory: maximal dpLimit overshoot, maximal dpTolerance overshoot, maximal
        deviation of the norm from 1 (mcwf::Logger)."""
        a = np.zeros(self.n_traj)
        b = np.zeros(self.n_traj)
        c = np.zeros(self.n_traj)
        P = C.POINTER(C.c_double)
        check(lib().cqg_ensemble_get_logger_maxima(self._h, a.ctypes.data_as(P), b.ctypes.data_as(P),
                                                   c.ctypes.data_as(P)))
        return a, b, c

    def jumps(self, i, cap=64):
        t = np.zeros(cap)
        l = np.zeros(cap, dtype=np.int32)
        n = C.c_int32()
        check(lib().cqg_ensemble_get_jumps(self._h, int(i), cap, t.ctypes.data_as(C.POINTER(C.c_double)),
                                           l.ctypes.data_as(C.POINTER(C.c_int32)), C.byref(n)))
        return t[:n.value], l[:n.value]

    def set_jump_capacity(self, cap):
        """Per-trajectory capacity of the jump record rings (default 64)."""
        check(lib().cqg_ensemble_set_jump_capacity(self._h, int(cap)))

    def jump_rings(self):
        """(counts [n_traj], times [n_traj, cap], lindblads [n_traj, cap]): every ring at once;
        the k-th jump of trajectory i is at slot k % cap while k >= counts[i] - cap."""
        cap = C.c_int32()
        check(lib().cqg_ensemble_get_jump_rings(self._h, C.byref(cap), None, None, None))
        counts = np.zeros(self.n_traj, dtype=np.uint64)
        times = np.zeros((self.n_traj, cap.value))
        lind = np.zeros((self.n_traj, cap.value), dtype=np.int32)
        check(lib().cqg_ensemble_get_jump_rings(self._h, None, counts.ctypes.data_as(C.POINTER(C.c_uint64)),
                                                times.ctypes.data_as(C.POINTER(C.c_double)),
                                                lind.ctypes.data_as(C.POINTER(C.c_int32))))
        return counts, times, lind

    def status(self):
        b = C.c_uint32()
        rc = lib().cqg_ensemble_status(self._h, C.byref(b))
        return rc, b.value

    def last_ms(self):
        """(kernel, whole call) device milliseconds of the last run call."""
        k = C.c_double()
        r = C.c_double()
        check(lib().cqg_ensemble_last_kernel_ms(self._h, C.byref(k), C.byref(r)))
        return k.value, r.value

    def save(self):
        """Checkpoint of every trajectory (bytes), see cqg_ensemble_save."""
        n = C.c_uint64()
        check(lib().cqg_ensemble_save(self._h, None, 0, C.byref(n)))
        buf = C.create_string_buffer(n.value)
        check(lib().cqg_ensemble_save(self._h, buf, n.value, C.byref(n)))
        return buf.raw

    def load(self, state):
        check(lib().cqg_ensemble_load(self._h, C.c_char_p(state), len(state)))

    def plan(self):
        """Kernel groups: list of dicts (kind, E, smax, threads, count)."""
        n = C.c_int32()
        check(lib().cqg_ensemble_plan(self._h, C.byref(n), None, 0))
        buf = (C.c_int32 * (5 * max(n.value, 1)))()
        check(lib().cqg_ensemble_plan(self._h, C.byref(n), buf, n.value))
        keys = ("kind", "E", "smax", "threads", "count")
        return [dict(zip(keys, buf[5 * g:5 * g + 5])) for g in range(n.value)]


def probe_fma_peaks():
    """Measured FP64 and FP32 FMA throughput (TFLOP/s) of the current device."""
    a = C.c_double()
    b = C.c_double()
    check(lib().cqg_probe_fma_peaks(C.byref(a), C.byref(b)))
    return a.value, b.value


class Master:
    """Master equation on the device (cqg_master_*); rho starts as |psi0><psi0|."""

    def __init__(self, system, psi0, pars):
        self._keep = system
        self.n_avr = None
        buf, _keep = to_c(psi0)
        self.dim = len(psi0)
        h = C.c_void_p()
        check(lib().cqg_master_create(system._h, buf, C.byref(pars), C.byref(h)))
        self._h = h

    def __del__(self):
        if getattr(self, "_h", None):
            lib().cqg_master_destroy(self._h)
            self._h = None

    def _buf(self, rows, n_avr):
        return np.zeros((rows, n_avr + 1))

    def run(self, Dt, n_intervals, n_avr):
        """Expectation values (n_avr linear averages, then dtDid) after each interval."""
        out = self._buf(n_intervals, n_avr)
        check(lib().cqg_master_run(self._h, float(Dt), int(n_intervals), out.ctypes.data_as(C.POINTER(C.c_double))))
        return out

    def steps(self, n_steps, T, n_avr):
        out = self._buf(1, n_avr)
        check(lib().cqg_master_steps(self._h, int(n_steps), float(T), out.ctypes.data_as(C.POINTER(C.c_double))))
        return out[0]

    def rho(self):
        r = np.zeros((self.dim, self.dim), dtype=np.complex128)
        check(lib().cqg_master_get_rho(self._h, r.ctypes.data_as(C.POINTER(A.cqg_complex))))
        return r

    def times(self):
        t, did, tr = C.c_double(), C.c_double(), C.c_double()
        check(lib().cqg_master_get_times(self._h, C.byref(t), C.byref(did), C.byref(tr)))
        return t.value, did.value, tr.value


class Server:
    """Continuous-batching request server (cqg_server_*)."""

    def __init__(self, pars=None, hbm_budget_bytes=None, max_trajectories=None, max_averages=None):
        p = A.cqg_server_pars()
        lib().cqg_server_pars_default(C.byref(p))
        if pars is not None:
            p.mcwf = pars
        if hbm_budget_bytes is not None:
            p.hbm_budget_bytes = int(hbm_budget_bytes)
        if max_trajectories is not None:
            p.max_trajectories = int(max_trajectories)
        if max_averages is not None:
            p.max_averages = int(max_averages)
        h = C.c_void_p()
        check(lib().cqg_server_create(C.byref(p), C.byref(h)))
        self._h = h
        self._keep = []

    def __del__(self):
        if getattr(self, "_h", None):
            lib().cqg_server_destroy(self._h)
            self._h = None

    def submit(self, system, psi0, n_traj, T, Dt, prng_stream):
        self._keep.append(system)
        buf, _keep = to_c(psi0)
        rid = C.c_int64()
        check(lib().cqg_server_submit(self._h, system._h, buf, int(n_traj), float(T), float(Dt), int(prng_stream),
                                      C.byref(rid)))
        return rid.value

    def round(self):
        a = C.c_int32()
        w = C.c_int32()
        check(lib().cqg_server_round(self._h, C.byref(a), C.byref(w)))
        return a.value, w.value

    def completed(self):
        n = C.c_int32()
        check(lib().cqg_server_completed(self._h, None, 0, C.byref(n)))
        ids = (C.c_int64 * max(n.value, 1))()
        check(lib().cqg_server_completed(self._h, ids, n.value, C.byref(n)))
        return list(ids[:n.value])

    def result(self, rid):
        """(rows [n_rows, n_avr + 1] of ensemble sums, accepted steps, (submit, admit, done) s, status)."""
        nr = C.c_int32()
        nc = C.c_int32()
        check(lib().cqg_server_result(self._h, int(rid), None, 0, C.byref(nr), C.byref(nc), None, None, None))
        rows = np.zeros((nr.value, nc.value))
        steps = C.c_uint64()
        times = (C.c_double * 3)()
        st = C.c_uint32()
        check(lib().cqg_server_result(self._h, int(rid), rows.ctypes.data_as(C.POINTER(C.c_double)), nr.value,
                                      C.byref(nr), C.byref(nc), C.byref(steps), times, C.byref(st)))
        return rows, steps.value, tuple(times), st.value

    def stats(self):
        s = C.c_uint64()
        ms = C.c_double()
        r = C.c_int64()
        check(lib().cqg_server_stats(self._h, C.byref(s), C.byref(ms), C.byref(r)))
        return s.value, ms.value, r.value
