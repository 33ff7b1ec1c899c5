"""ctypes mirror of include/cqg.h and include/cqg_model.h.

Only layouts and prototypes live here; loading the libraries is done by
:mod:`cppqed_b200.engine`.
"""
import ctypes as C

MAX_RANK = 8

CQG_OK = 0
CQG_E_INVALID = -1
CQG_E_CUDA = -2
CQG_E_NOMEM = -3
CQG_E_UNSUPPORTED = -4
CQG_E_NONFINITE = -5
CQG_E_STALLED = -6
CQG_E_NODEVICE = -7

RNG_PCG64 = 0
RNG_PHILOX = 1
FP64 = 0
FP32 = 1

EVOL_SINGLE = 0
EVOL_ENSEMBLE = 1
EVOL_MASTER = 2


class cqg_complex(C.Structure):
    _fields_ = [("re", C.c_double), ("im", C.c_double)]


class cqg_tridiagonal(C.Structure):
    _fields_ = [
        ("rank", C.c_int32),
        ("axes", C.c_int32 * MAX_RANK),
        ("differences", C.c_int64 * MAX_RANK),
        ("diagonals", C.POINTER(C.POINTER(cqg_complex))),
        ("freqs", C.POINTER(C.POINTER(cqg_complex))),
    ]


class cqg_jump(C.Structure):
    _fields_ = [
        ("op", cqg_tridiagonal),
        ("rate_axis", C.c_int32),
        ("rate_weights", C.POINTER(C.c_double)),
    ]


class cqg_observable(C.Structure):
    _fields_ = [
        ("op", cqg_tridiagonal),
        ("dense", C.POINTER(cqg_complex)),
        ("dense_axis", C.c_int32),
        ("col_re", C.c_int32),
        ("col_im", C.c_int32),
        ("fourier", C.c_int32),
        ("reserved", C.c_int32),
        ("fourier_weights", C.POINTER(C.c_double)),
    ]


class cqg_system_desc(C.Structure):
    _fields_ = [
        ("rank", C.c_int32),
        ("dims", C.c_int64 * MAX_RANK),
        ("n_ham", C.c_int32),
        ("ham", C.POINTER(cqg_tridiagonal)),
        ("has_hamiltonian", C.c_int32),
        ("exact", C.POINTER(cqg_complex) * MAX_RANK),
        ("n_jumps", C.c_int32),
        ("jumps", C.POINTER(cqg_jump)),
        ("n_obs", C.c_int32),
        ("obs", C.POINTER(cqg_observable)),
        ("n_avr", C.c_int32),
        ("highest_frequency", C.c_double),
    ]


class cqg_mcwf_pars(C.Structure):
    _fields_ = [
        ("eps_rel", C.c_double),
        ("eps_abs", C.c_double),
        ("dp_limit", C.c_double),
        ("overshoot_tolerance", C.c_double),
        ("dt_init", C.c_double),
        ("seed", C.c_uint64),
        ("prng_stream", C.c_uint64),
        ("rng", C.c_int32),
        ("noise", C.c_int32),
        ("precision", C.c_int32),
        ("max_attempts", C.c_int32),
        ("autotune", C.c_int32),
        ("cta_threads", C.c_int32),
        ("cta_shared_vectors", C.c_int32),
        ("ip_phase_table", C.c_int32),
        ("yield_steps", C.c_int32),
    ]


class cqg_server_pars(C.Structure):
    _fields_ = [
        ("hbm_budget_bytes", C.c_uint64),
        ("max_trajectories", C.c_int32),
        ("max_systems", C.c_int32),
        ("max_averages", C.c_int32),
        ("reserved", C.c_int32),
        ("mcwf", cqg_mcwf_pars),
    ]


class cqg_run_pars(C.Structure):
    _fields_ = [
        ("T", C.c_double),
        ("Dt", C.c_double),
        ("dc", C.c_int32),
        ("NDt", C.c_int64),
        ("sdf", C.c_int32),
        ("n_traj", C.c_int64),
        ("evol", C.c_int32),
        ("log_level", C.c_int32),
        ("mcwf", cqg_mcwf_pars),
    ]


_P = C.c_void_p
_DP = C.POINTER(C.c_double)
_CP = C.POINTER(cqg_complex)

# name -> (restype, argtypes); every symbol declared in include/cqg.h and include/cqg_model.h
ENGINE_PROTOTYPES = {
    "cqg_last_error": (C.c_char_p, []),
    "cqg_abi_version": (C.c_int, []),
    "cqg_mcwf_pars_default": (None, [C.POINTER(cqg_mcwf_pars)]),
    "cqg_device_count": (C.c_int, [C.POINTER(C.c_int)]),
    "cqg_system_create": (C.c_int, [C.POINTER(cqg_system_desc), C.POINTER(_P)]),
    "cqg_system_dimension": (C.c_int, [_P, C.POINTER(C.c_int64)]),
    "cqg_system_destroy": (C.c_int, [_P]),
    "cqg_system_apply_hamiltonian": (C.c_int, [_P, C.c_void_p, C.c_void_p, C.c_int64, C.c_double, C.c_void_p]),
    "cqg_ensemble_create": (C.c_int, [_P, _CP, C.c_int64, C.POINTER(cqg_mcwf_pars), C.POINTER(_P)]),
    "cqg_batch_create": (C.c_int, [C.POINTER(_P), C.c_int32, C.POINTER(C.c_int32), _CP,
                                   C.POINTER(C.c_int64), C.c_int64, C.POINTER(cqg_mcwf_pars),
                                   C.POINTER(_P)]),
    "cqg_ensemble_run": (C.c_int, [_P, C.c_double, C.c_int32, _DP]),
    "cqg_ensemble_advance_to": (C.c_int, [_P, C.c_double, _DP]),
    "cqg_ensemble_steps": (C.c_int, [_P, C.c_int32, C.c_double, _DP]),
    "cqg_ensemble_traj_averages": (C.c_int, [_P, _DP]),
    "cqg_ensemble_size": (C.c_int, [_P, C.POINTER(C.c_int64), C.POINTER(C.c_int32)]),
    "cqg_ensemble_get_state": (C.c_int, [_P, C.c_int64, _CP]),
    "cqg_ensemble_set_state": (C.c_int, [_P, C.c_int64, _CP]),
    "cqg_ensemble_get_times": (C.c_int, [_P, _DP, _DP, _DP]),
    "cqg_ensemble_get_counters": (C.c_int, [_P, C.POINTER(C.c_uint64)]),
    "cqg_ensemble_get_logger_maxima": (C.c_int, [_P, _DP, _DP, _DP]),
    "cqg_ensemble_get_jumps": (C.c_int, [_P, C.c_int64, C.c_int32, _DP, C.POINTER(C.c_int32),
                                         C.POINTER(C.c_int32)]),
    "cqg_ensemble_get_jump_rings": (C.c_int, [_P, C.POINTER(C.c_int32), C.POINTER(C.c_uint64), _DP,
                                              C.POINTER(C.c_int32)]),
    "cqg_ensemble_set_jump_capacity": (C.c_int, [_P, C.c_int32]),
    "cqg_ensemble_status": (C.c_int, [_P, C.POINTER(C.c_uint32)]),
    "cqg_ensemble_last_kernel_ms": (C.c_int, [_P, _DP, _DP]),
    "cqg_ensemble_save": (C.c_int, [_P, C.c_void_p, C.c_uint64, C.POINTER(C.c_uint64)]),
    "cqg_ensemble_load": (C.c_int, [_P, C.c_void_p, C.c_uint64]),
    "cqg_ensemble_plan": (C.c_int, [_P, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.c_int32]),
    "cqg_probe_fma_peaks": (C.c_int, [_DP, _DP]),
    "cqg_master_create": (C.c_int, [_P, _CP, C.POINTER(cqg_mcwf_pars), C.POINTER(_P)]),
    "cqg_master_run": (C.c_int, [_P, C.c_double, C.c_int32, _DP]),
    "cqg_master_steps": (C.c_int, [_P, C.c_int32, C.c_double, _DP]),
    "cqg_master_averages": (C.c_int, [_P, _DP]),
    "cqg_master_get_rho": (C.c_int, [_P, _CP]),
    "cqg_master_get_times": (C.c_int, [_P, _DP, _DP, _DP]),
    "cqg_master_destroy": (C.c_int, [_P]),
    "cqg_server_pars_default": (None, [C.POINTER(cqg_server_pars)]),
    "cqg_server_create": (C.c_int, [C.POINTER(cqg_server_pars), C.POINTER(_P)]),
    "cqg_server_submit": (C.c_int, [_P, _P, _CP, C.c_int64, C.c_double, C.c_double, C.c_uint64,
                                    C.POINTER(C.c_int64)]),
    "cqg_server_round": (C.c_int, [_P, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "cqg_server_completed": (C.c_int, [_P, C.POINTER(C.c_int64), C.c_int32, C.POINTER(C.c_int32)]),
    "cqg_server_result": (C.c_int, [_P, C.c_int64, _DP, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                    C.POINTER(C.c_uint64), _DP, C.POINTER(C.c_uint32)]),
    "cqg_server_stats": (C.c_int, [_P, C.POINTER(C.c_uint64), _DP, C.POINTER(C.c_int64)]),
    "cqg_server_destroy": (C.c_int, [_P]),
    "cqg_ensemble_destroy": (C.c_int, [_P]),
    "cqg_system_averages_noalloc": (C.c_int, [_P, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p]),
    "cqg_model_create": (C.c_int, [C.c_char_p, C.c_int32, C.POINTER(C.c_char_p), C.POINTER(_P)]),
    "cqg_model_desc": (C.c_int, [_P, C.POINTER(C.POINTER(cqg_system_desc))]),
    "cqg_model_dimension": (C.c_int, [_P, C.POINTER(C.c_int64)]),
    "cqg_model_initial_state": (C.c_int, [_P, _CP]),
    "cqg_model_run_pars": (C.c_int, [_P, C.POINTER(cqg_run_pars)]),
    "cqg_model_n_avr": (C.c_int, [_P, C.POINTER(C.c_int32)]),
    "cqg_model_process": (C.c_int, [_P, _DP]),
    "cqg_model_key": (C.c_int, [_P, C.c_char_p, C.c_size_t]),
    "cqg_model_key_text": (C.c_int, [_P, C.c_int32, C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t)]),
    "cqg_model_parameters_text": (C.c_int, [_P, C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t)]),
    "cqg_model_command_line": (C.c_int, [_P, C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t)]),
    "cqg_model_destroy": (C.c_int, [_P]),
}

def bind(lib, prototypes):
    for name, (res, args) in prototypes.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib
