"""The allocation-free averages entry point against the ensemble path.

cqg_system_averages_noalloc exists for callers that cannot allocate device memory
(their memory belongs to another allocator, or cudaMalloc is not allowed where they
run).  It reads caller-owned device states and writes caller-owned device sums, keeping
its intermediate per-state sums in a fixed device array.  Here it must give the same
ensemble sums as cqg_ensemble_steps(n_steps=0) on the same states, on two calls in a row
(the second with fewer states, so nothing may carry over from the first), on the default
stream and on a caller's stream, for a Schroedinger-picture system, an interaction-picture
system whose states come from a running ensemble (at t0 = t), and a particle in a cavity
with dense position observables.  It must refuse requests larger than its fixed array and
misaligned pointers.  This file sorts last so a stop-at-first-failure run has executed
every other test before it.
"""
import ctypes as C

import numpy as np
import pytest

from cppqed_b200 import _abi as A

pytestmark = pytest.mark.gpu

ARGS = ["--picture", "Sch", "--deltaA", "0", "--gamma", "0.5", "--deltaC", "0", "--kappa", "1",
        "--eta", "1.5", "--cutoff", "40", "--g", "2"]
IP_ARGS = ["--picture", "IP", "--deltaA", "-1", "--gamma", "0.5", "--deltaC", "2", "--kappa", "1",
           "--eta", "1.5", "--cutoff", "40", "--g", "2"]
PARTICLE_ARGS = ["--1p1mconf", "2", "--vClass", "0", "--modeCav", "Cos", "--kCav", "1", "--Unot", "-1",
                 "--eta", "5", "--kappa", "1", "--cutoff", "8", "--fin", "5"]

# (script, args, where the states come from, stream)
CASES = {
    "qbitmode_sch_random_default_stream": ("QbitMode_C++QED", ARGS, "random", "default"),
    "qbitmode_ip_ensemble_states_own_stream": ("QbitMode_C++QED", IP_ARGS, "ensemble", "own"),
    "particle_cavity_dense_obs_own_stream": ("1particle1mode", PARTICLE_ARGS, "ensemble", "own"),
}


def random_states(n, dim, seed):
    rng = np.random.default_rng(seed)
    psi = rng.normal(size=(n, dim)) + 1j * rng.normal(size=(n, dim))
    psi /= np.linalg.norm(psi, axis=1, keepdims=True)
    return psi.astype(np.complex128)


def evolved_states(gpu, system, model, n, seed):
    """States of an ensemble after two output intervals (the picture's frame at t0 = t)."""
    pars = model.run_pars().mcwf
    pars.prng_stream = seed
    ens = gpu.Ensemble(system, model.initial_state(), n, pars)
    ens.run(0.1, 2)
    return np.stack([ens.state(i, model.dim) for i in range(n)])


def ensemble_sums(gpu, system, model, psi):
    pars = model.run_pars().mcwf
    pars.precision = A.FP64
    ens = gpu.Ensemble(system, psi[0], len(psi), pars)
    for i, p in enumerate(psi):
        ens.set_state(i, p)
    return ens.steps(0, 1.0)[:model.n_avr]


@pytest.mark.parametrize("case", sorted(CASES))
def test_noalloc_averages_match_ensemble_path_twice(gpu, case):
    import torch

    script, args, source, where = CASES[case]
    model = gpu.Model(script, args)
    system = gpu.System(model.desc)
    lib = gpu.lib()
    stream = torch.cuda.Stream() if where == "own" else None
    for n, seed in ((300, 1), (100, 2)):
        if source == "random":
            psi = random_states(n, model.dim, seed)
        else:
            psi = evolved_states(gpu, system, model, n // 4, seed)
        d_psi = torch.from_numpy(psi).to("cuda")
        d_sums = torch.full((model.n_avr,), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        handle = C.c_void_p(stream.cuda_stream) if stream is not None else None
        rc = lib.cqg_system_averages_noalloc(system._h, C.c_void_p(d_psi.data_ptr()), len(psi),
                                             C.c_void_p(d_sums.data_ptr()), handle)
        assert rc == A.CQG_OK, lib.cqg_last_error()
        torch.cuda.synchronize()
        got = d_sums.cpu().numpy()
        ref = ensemble_sums(gpu, system, model, psi)
        # per-state rounding (the particle's position moments: dense matrix here, a fast
        # transform on the ensemble path) summed over the states
        assert np.allclose(got, ref, rtol=1e-11, atol=1e-13 * len(psi)), (got, ref)


def test_noalloc_averages_reject_oversized_requests(gpu):
    import torch

    model = gpu.Model("QbitMode_C++QED", ARGS)
    system = gpu.System(model.desc)
    lib = gpu.lib()
    d_psi = torch.zeros(model.dim, dtype=torch.complex128, device="cuda")
    d_sums = torch.zeros(model.n_avr, dtype=torch.float64, device="cuda")
    too_many = (1 << 18) // model.n_avr + 1
    rc = lib.cqg_system_averages_noalloc(system._h, C.c_void_p(d_psi.data_ptr()), too_many,
                                         C.c_void_p(d_sums.data_ptr()), None)
    assert rc == A.CQG_E_INVALID
    assert b"exceeds the fixed scratch" in lib.cqg_last_error()


def test_noalloc_averages_reject_misaligned_pointers(gpu):
    """States are read as 16-byte complex vectors and sums written as doubles: pointers off
    those boundaries are refused on the host, before any work reaches the GPU."""
    import torch

    model = gpu.Model("QbitMode_C++QED", ARGS)
    system = gpu.System(model.desc)
    lib = gpu.lib()
    d_psi = torch.zeros(2 * model.dim + 1, dtype=torch.complex128, device="cuda")
    d_sums = torch.zeros(model.n_avr + 1, dtype=torch.float64, device="cuda")
    rc = lib.cqg_system_averages_noalloc(system._h, C.c_void_p(d_psi.data_ptr() + 8), 1,
                                         C.c_void_p(d_sums.data_ptr()), None)
    assert rc == A.CQG_E_INVALID
    assert b"16-byte aligned" in lib.cqg_last_error()
    rc = lib.cqg_system_averages_noalloc(system._h, C.c_void_p(d_psi.data_ptr()), 1,
                                         C.c_void_p(d_sums.data_ptr() + 4), None)
    assert rc == A.CQG_E_INVALID
    assert b"8-byte aligned" in lib.cqg_last_error()
