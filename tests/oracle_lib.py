"""Test-side access to the CPU oracle (oracle/_build/liboracle.so).

The oracle is the checker: a restatement of the reference's MCWF path that the
device results are compared with.  Nothing in the engine imports this module."""
import ctypes as C
import os
import subprocess
import sys

import numpy as np

from cppqed_b200 import _abi as A

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PATH = os.path.join(ROOT, "oracle", "_build", "liboracle.so")

_CP = C.POINTER(A.cqg_complex)
_DP = C.POINTER(C.c_double)

# C prototypes of the oracle library (oracle/oracle.cpp)
ORACLE_PROTOTYPES = {
    "oracle_last_error": (C.c_char_p, []),
    "oracle_pcg64_uniform": (C.c_int, [C.c_uint64, C.c_uint64, C.c_int64, _DP]),
    "oracle_pcg64_state_text": (C.c_int, [C.c_uint64, C.c_uint64, C.c_int64, C.c_char_p, C.c_size_t]),
    "oracle_apply_hamiltonian": (C.c_int, [C.POINTER(A.cqg_system_desc), _CP, C.c_double, _CP]),
    "oracle_run": (C.c_int, [C.POINTER(A.cqg_system_desc), _CP, C.POINTER(A.cqg_run_pars), _DP, C.c_int64,
                             C.POINTER(C.c_int64), _CP]),
    "oracle_trajectory": (C.c_int, [C.POINTER(A.cqg_system_desc), _CP, C.POINTER(A.cqg_mcwf_pars), C.c_uint64,
                                    C.c_double, C.c_int64, C.c_double, _CP, _DP, C.POINTER(C.c_uint64),
                                    _DP, C.POINTER(C.c_int32), C.c_int64, C.POINTER(C.c_int64)]),
    "oracle_ensemble_bench": (C.c_int, [C.POINTER(A.cqg_system_desc), _CP, C.POINTER(A.cqg_mcwf_pars), C.c_int64,
                                        C.c_double, C.c_int64, C.c_int64, C.c_int32, C.c_int32,
                                        C.POINTER(C.c_uint64), _DP, _DP]),
}


def build_oracle(verbose=False):
    """Builds the CPU oracle with its Makefile (oracle/_build/liboracle.so)."""
    cmd = ["make", "-s", "-C", os.path.join(ROOT, "oracle"), "PYTHON=" + sys.executable]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("oracle build failed")
    return PATH


class Oracle:
    def __init__(self):
        self.lib = A.bind(C.CDLL(PATH), ORACLE_PROTOTYPES)

    def _err(self):
        return self.lib.oracle_last_error().decode()

    def run(self, model, run_pars=None, final_state=False):
        """trajectory::run of the model's --evol; rows (t, dtDid, processed averages)."""
        rp = run_pars or model.run_pars()
        n = model.n_avr
        cap = 200000
        rows = np.zeros(cap * (2 + n))
        nr = C.c_int64()
        psi = model.initial_state()
        D = model.dim
        fs = None
        if final_state:
            fs = np.zeros(D if rp.evol == A.EVOL_SINGLE else D * D, dtype=np.complex128)
        rc = self.lib.oracle_run(model.desc, psi.ctypes.data_as(C.POINTER(A.cqg_complex)), C.byref(rp),
                                 rows.ctypes.data_as(C.POINTER(C.c_double)), cap, C.byref(nr),
                                 fs.ctypes.data_as(C.POINTER(A.cqg_complex)) if fs is not None else None)
        if rc:
            raise RuntimeError(self._err())
        R = rows[:nr.value * (2 + n)].reshape(nr.value, 2 + n).copy()
        for r in R:
            r[2:] = model.process(r[2:])
        return (R, fs) if final_state else R

    def trajectory(self, model, pars, stream, Dt, n_intervals, T=0.0, psi0=None, jump_cap=4096):
        """One trajectory advanced n_intervals x Dt (Dt <= 0: n_intervals steps of T - t)."""
        D = model.dim
        psi = model.initial_state() if psi0 is None else np.ascontiguousarray(psi0, dtype=np.complex128)
        out = np.zeros(D, dtype=np.complex128)
        times = np.zeros(3)
        cnt = np.zeros(8, dtype=np.uint64)
        jt = np.zeros(jump_cap)
        jl = np.zeros(jump_cap, dtype=np.int32)
        nj = C.c_int64()
        P = C.POINTER(A.cqg_complex)
        rc = self.lib.oracle_trajectory(model.desc, psi.ctypes.data_as(P), C.byref(pars), int(stream), float(Dt),
                                        int(n_intervals), float(T), out.ctypes.data_as(P),
                                        times.ctypes.data_as(C.POINTER(C.c_double)),
                                        cnt.ctypes.data_as(C.POINTER(C.c_uint64)),
                                        jt.ctypes.data_as(C.POINTER(C.c_double)),
                                        jl.ctypes.data_as(C.POINTER(C.c_int32)), jump_cap, C.byref(nj))
        if rc:
            raise RuntimeError(self._err())
        k = min(nj.value, jump_cap)
        return {"psi": out, "t": times[0], "dtDid": times[1], "dtTry": times[2], "counters": cnt,
                "jump_t": jt[:k], "jump_l": jl[:k]}

    def apply_hamiltonian(self, model, psi, tau=0.0):
        psi = np.ascontiguousarray(psi, dtype=np.complex128)
        out = np.zeros_like(psi)
        P = C.POINTER(A.cqg_complex)
        if self.lib.oracle_apply_hamiltonian(model.desc, psi.ctypes.data_as(P), float(tau), out.ctypes.data_as(P)):
            raise RuntimeError(self._err())
        return out

    def pcg64_uniform(self, seed, stream, n):
        out = np.zeros(n)
        self.lib.oracle_pcg64_uniform(seed, stream, n, out.ctypes.data_as(C.POINTER(C.c_double)))
        return out

    def pcg64_state_text(self, seed, stream, n_draws=0):
        buf = C.create_string_buffer(256)
        self.lib.oracle_pcg64_state_text(seed, stream, n_draws, buf, 256)
        return buf.value.decode()

    def ensemble_bench(self, model, pars, n_traj, Dt, n_intervals, threads=1, with_rho=True, warm_intervals=0):
        """The reference's serial ensemble on n_traj trajectories: warm_intervals untimed
        intervals of Dt, then n_intervals timed ones.  (steps, seconds, sums per interval) of
        the timed part."""
        steps = C.c_uint64()
        secs = C.c_double()
        sums = np.zeros(n_intervals * model.n_avr)
        psi = model.initial_state()
        rc = self.lib.oracle_ensemble_bench(model.desc, psi.ctypes.data_as(C.POINTER(A.cqg_complex)), C.byref(pars),
                                            int(n_traj), float(Dt), int(warm_intervals), int(n_intervals),
                                            int(threads), int(with_rho), C.byref(steps), C.byref(secs),
                                            sums.ctypes.data_as(C.POINTER(C.c_double)))
        if rc:
            raise RuntimeError(self._err())
        return steps.value, secs.value, sums.reshape(n_intervals, model.n_avr)
