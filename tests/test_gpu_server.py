"""The request server (continuous batching): a request's result is the same alone, in a
mix with requests of other systems and kernel shapes that arrive before and after it, and
as a plain ensemble on the same random streams; admission waits for slots and state memory
to free up."""
import numpy as np
import pytest

from cppqed_b200 import _abi as A

pytestmark = pytest.mark.gpu

QM = ["--picture", "Sch", "--deltaA", "0", "--gamma", "0.5", "--deltaC", "0", "--kappa", "1",
      "--eta", "1.5", "--cutoff", "40", "--g", "2"]
PLM = ["--picture", "Sch", "--deltaC", "-1", "--eta", "2", "--kappa", "1", "--cutoff", "30", "--no_quadratures"]
OPTO = ["--picture", "Sch", "--cutoffOpt", "15", "--cutoffMech", "30", "--etaOpt", "2", "--kappaOpt", "1",
        "--deltaCOpt", "-1", "--kappaMech", "0.1", "--deltaCMech", "-2", "--u", "0.2"]
T, DT = 0.5, 0.125


def _setup(gpu, script, args):
    m = gpu.Model(script, args)
    return m, gpu.System(m.desc)


def _alone_rows(gpu, model, system, n, stream):
    pars = model.run_pars().mcwf
    pars.prng_stream = stream
    ens = gpu.Ensemble(system, model.initial_state(), n, pars)
    return np.concatenate([ens.run(DT, 1) for _ in range(int(T / DT))])


def _drain(srv):
    rounds = 0
    while True:
        active, waiting = srv.round()
        rounds += 1
        assert rounds < 1000
        if active == 0 and waiting == 0:
            return


def test_request_alone_equals_plain_ensemble(gpu):
    model, system = _setup(gpu, "QbitMode_C++QED", QM)
    srv = gpu.Server(model.run_pars().mcwf)
    rid = srv.submit(system, model.initial_state(), 100, T, DT, 7)
    _drain(srv)
    assert srv.completed() == [rid]
    rows, steps, times, status = srv.result(rid)
    assert status == 0 and steps > 0 and times[0] <= times[1] <= times[2]
    ref = _alone_rows(gpu, model, system, 100, 7)
    assert rows.shape == ref.shape == (4, model.n_avr + 1)
    assert np.array_equal(rows, ref)


def test_request_result_is_the_same_in_a_mix(gpu):
    """Requests of three systems (warp kernel D = 80 and 30, CTA kernel D = 450) admitted
    in different rounds share launches; each result equals its request alone."""
    qm, s_qm = _setup(gpu, "QbitMode_C++QED", QM)
    plm, s_plm = _setup(gpu, "PumpedLossyMode_C++QED", PLM)
    opt, s_opt = _setup(gpu, "Optomechanics", OPTO)
    srv = gpu.Server(qm.run_pars().mcwf)
    ids = {}
    ids["qm"] = srv.submit(s_qm, qm.initial_state(), 100, T, DT, 7)
    ids["opt"] = srv.submit(s_opt, opt.initial_state(), 24, T, DT, 1001)
    srv.round()
    ids["plm"] = srv.submit(s_plm, plm.initial_state(), 300, T, DT, 50)
    srv.round()
    ids["qm2"] = srv.submit(s_qm, qm.initial_state(), 64, T, DT, 500)
    _drain(srv)
    assert sorted(srv.completed()) == sorted(ids.values())
    cases = {"qm": (qm, s_qm, 100, 7), "opt": (opt, s_opt, 24, 1001), "plm": (plm, s_plm, 300, 50),
             "qm2": (qm, s_qm, 64, 500)}
    for name, (m, s, n, stream) in cases.items():
        rows, _, _, status = srv.result(ids[name])
        assert status == 0
        assert np.array_equal(rows, _alone_rows(gpu, m, s, n, stream)), name


def test_admission_waits_for_memory(gpu):
    """With slots for only one of two requests, the second is admitted after the first
    retires and still gives its alone result."""
    model, system = _setup(gpu, "QbitMode_C++QED", QM)
    srv = gpu.Server(model.run_pars().mcwf, max_trajectories=128)
    a = srv.submit(system, model.initial_state(), 100, T, DT, 7)
    b = srv.submit(system, model.initial_state(), 100, T, DT, 300)
    active, waiting = srv.round()
    assert (active, waiting) == (1, 1)
    _drain(srv)
    ra = srv.result(a)
    rb = srv.result(b)
    assert rb[2][1] >= ra[2][2]  # b admitted after a finished
    assert np.array_equal(rb[0], _alone_rows(gpu, model, system, 100, 300))


def test_request_larger_than_the_server_is_refused(gpu):
    model, system = _setup(gpu, "QbitMode_C++QED", QM)
    srv = gpu.Server(model.run_pars().mcwf, max_trajectories=64)
    with pytest.raises(gpu.EngineError) as e:
        srv.submit(system, model.initial_state(), 65, T, DT, 1)
    assert e.value.code == A.CQG_E_INVALID
