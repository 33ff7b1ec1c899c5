"""The allocation-free averages entry point against the ensemble path.

cqg_system_averages_noalloc exists for callers that cannot allocate device memory
(their memory belongs to another allocator, or cudaMalloc is not allowed where they
run).  It reads caller-owned device states and writes caller-owned device sums, keeping
its intermediate per-state sums in a fixed device array.  Here it must give the same
ensemble sums as cqg_ensemble_steps(n_steps=0) on the same states, on two calls in a row
(the second with fewer states, so nothing may carry over from the first), and it must
refuse requests larger than its fixed array.  This file sorts last so a stop-at-first-
failure run has executed every other test before it.
"""
import ctypes as C

import numpy as np
import pytest

from cppqed_b200 import _abi as A

pytestmark = pytest.mark.gpu

ARGS = ["--picture", "Sch", "--deltaA", "0", "--gamma", "0.5", "--deltaC", "0", "--kappa", "1",
        "--eta", "1.5", "--cutoff", "40", "--g", "2"]


def random_states(n, dim, seed):
    rng = np.random.default_rng(seed)
    psi = rng.normal(size=(n, dim)) + 1j * rng.normal(size=(n, dim))
    psi /= np.linalg.norm(psi, axis=1, keepdims=True)
    return psi.astype(np.complex128)


def ensemble_sums(gpu, system, model, psi):
    pars = model.run_pars().mcwf
    pars.precision = A.FP64
    ens = gpu.Ensemble(system, psi[0], len(psi), pars)
    for i, p in enumerate(psi):
        ens.set_state(i, p)
    return ens.steps(0, 1.0)[:model.n_avr]


def test_noalloc_averages_match_ensemble_path_twice(gpu):
    import torch

    model = gpu.Model("QbitMode_C++QED", ARGS)
    system = gpu.System(model.desc)
    lib = gpu.lib()
    for n, seed in ((300, 1), (100, 2)):
        psi = random_states(n, model.dim, seed)
        d_psi = torch.from_numpy(psi).to("cuda")
        d_sums = torch.full((model.n_avr,), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        rc = lib.cqg_system_averages_noalloc(system._h, C.c_void_p(d_psi.data_ptr()), n,
                                             C.c_void_p(d_sums.data_ptr()), None)
        assert rc == A.CQG_OK, lib.cqg_last_error()
        torch.cuda.synchronize()
        got = d_sums.cpu().numpy()
        ref = ensemble_sums(gpu, system, model, psi)
        assert np.allclose(got, ref, rtol=1e-12, atol=1e-13), (got, ref)


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
