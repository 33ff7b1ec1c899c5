"""The CPU oracle against the reference's own golden runs (Testing/expected, as
fixtures in tests/golden/reference_runs.json).  These pin the oracle: the Odeint
controller with its swapped eps arguments, the MCWF step, pcg64 streams, the run
loops, the ensemble density-operator average and the master equation."""
import numpy as np
import pytest

from cppqed_b200 import _abi as A

PTLA = ["run_PTLA_CPPQED_%s_%s" % (m, e) for m in ("dc", "dt", "ndt") for e in ("single", "ensemble", "master")]
# particle in a cavity (binary mode x particle, interaction picture, configurations 1-4 of
# ParticleOrthogonalToCavity / ParticleAlongCavity) and the ring cavity (composite
# particle x mode x mode with ParticleTwoModes)
PARTICLE = ["run_1particle1mode_%s_%s" % (m, e) for m in ("dc", "dt", "ndt", "ndt_conf2", "ndt_conf3", "ndt_conf4")
            for e in ("single", "ensemble", "master")]
RING = ["run_Ring_%s_%s" % (m, e) for m in ("dc", "dt", "ndt") for e in ("single", "ensemble", "master")]


@pytest.mark.parametrize("run", PTLA + PARTICLE + RING)
def test_golden(engine, oracle, golden, run):
    g = golden[run]
    model = engine.Model(g["script"], g["args"])
    rows = oracle.run(model)
    ref = np.array(g["rows"])
    assert rows.shape == ref.shape
    # testdriver.py Verifier._verify_ev: np.allclose on all streamed columns
    assert np.allclose(rows, ref)


def test_pcg64_seeding_matches_reference_archive(oracle, golden):
    # the first state archive of a single run holds the engine right after pcg64{1001, 1}
    state = golden["run_PTLA_CPPQED_dc_single"]["pcg64_first_archive"]
    assert oracle.pcg64_state_text(1001, 1) == state


def test_eps_arguments_are_swapped_as_in_the_reference(engine, oracle, golden):
    # make_controlled(epsRel, epsAbs, ...) puts epsRel into Odeint's absolute slot
    # (ODE.h:205); with the slots the other way round the dtDid column differs.
    g = golden["run_PTLA_CPPQED_dc_single"]
    model = engine.Model(g["script"], g["args"])
    rp = model.run_pars()
    rp.mcwf.eps_rel, rp.mcwf.eps_abs = rp.mcwf.eps_abs, rp.mcwf.eps_rel
    rows = oracle.run(model, rp)
    ref = np.array(g["rows"])
    assert rows.shape != ref.shape or not np.allclose(rows, ref)


def test_uniform_draws_are_canonical(oracle):
    u = oracle.pcg64_uniform(1001, 1, 10000)
    assert u.min() >= 0 and u.max() < 1
    assert abs(u.mean() - 0.5) < 0.02


def test_master_equation_fixture_is_the_oracle(oracle):
    """The bench states the error of the ensemble averages against the FP64 master equation
    held in tests/golden/master_equation_runs.json; it must be what the oracle computes."""
    import json
    import os

    import cppqed_b200 as cqg
    from cppqed_b200 import _abi as A

    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "master_equation_runs.json")
    runs = json.load(open(path))
    assert runs
    for name, r in runs.items():
        model = cqg.Model(r["script"], r["args"])
        rp = model.run_pars()
        rp.evol = A.EVOL_MASTER
        rp.dc = 0
        rp.T = r["T"]
        rp.Dt = r["Dt"]
        rp.NDt = 0
        rows = oracle.run(model, rp)
        assert model.key() == r["key"], name
        assert np.allclose(rows, np.array(r["rows"]), rtol=1e-13, atol=1e-15), name
