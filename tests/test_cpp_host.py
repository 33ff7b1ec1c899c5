"""The C++ host side (include/cqg_ensemble.hpp) and its driver program cqg_evolve.

cqg_evolve runs a workload script through the C ABI the way the reference's script does
(trajectory::run with its dc / Dt / NDt cadence) and writes the reference's trajectory file:
a '#'-commented header with the key to the columns, fixed-width rows, the end-of-run log.
The reference's own comparer (Testing/testdriver.py, Verifier._verify_ev) reads such files
with numpy.genfromtxt and compares them with numpy.allclose; so do these tests, against the
golden runs of the reference.
"""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from cppqed_b200 import _abi as A
from cppqed_b200 import build

EXE = os.path.join(build.LIBDIR, "cqg_evolve")


@pytest.fixture(scope="module")
def driver(engine):
    if not os.path.exists(EXE):
        build.build_apps()
    return EXE


def model_text(engine, fn, model, *args):
    lib = engine.lib()
    need = C.c_size_t()
    assert getattr(lib, fn)(model._h, *args, None, 0, C.byref(need)) == A.CQG_OK
    buf = C.create_string_buffer(need.value)
    assert getattr(lib, fn)(model._h, *args, buf, need.value, C.byref(need)) == A.CQG_OK
    return buf.value.decode()


def test_driver_builds_and_prints_usage(driver):
    r = subprocess.run([driver], capture_output=True, text=True)
    assert r.returncode == 2
    assert "usage: cqg_evolve" in r.stderr


@pytest.mark.parametrize("run", ["run_PTLA_CPPQED_dt_ensemble", "run_1particle1mode_ndt_ensemble",
                                 "run_1particle1mode_ndt_conf3_ensemble", "run_Ring_dt_ensemble"])
def test_key_text_matches_golden_headers(engine, golden, run):
    """The system's lines of the header's "Key to data" (element titles, numbered columns)
    are the reference's, line for line."""
    g = golden[run]
    model = engine.Model(g["script"], g["args"])
    key = model_text(engine, "cqg_model_key_text", model, C.c_int32(3)).splitlines()
    assert key == g["key"]


def read_trajectory_file(path):
    """Rows as the reference's testdriver loads them (numpy.genfromtxt skips '#' lines), and
    the end-of-run log lines."""
    rows = np.genfromtxt(path)
    log = [l[2:].rstrip("\n") for l in open(path) if l.startswith("# ")]
    return np.atleast_2d(rows), log


LOG_PATTERNS = {
    "average_steps": r"Average number of total steps: (\S+)",
    "average_overshot": r"On average, dpLimit overshot: (\S+) times",
    "max_overshoot": r"dpLimit overshot: \S+ times, maximal overshoot: (\S+)",
    "average_tolerance_overshot": r"On average, dpTolerance overshot: (\S+) times",
    "max_tolerance_overshoot": r"dpTolerance overshot: \S+ times, maximal overshoot: (\S+)",
    "max_norm_deviation": r"Maximal deviation of norm from 1: (\S+)",
    "average_jumps": r"Average number of total jumps: (\S+)",
}

GOLDEN_CPP = (["run_PTLA_CPPQED_%s_%s" % (m, e) for m in ("dc", "dt", "ndt") for e in ("single", "ensemble", "master")]
              + ["run_1particle1mode_ndt_ensemble", "run_1particle1mode_dc_single", "run_1particle1mode_dt_master",
                 "run_Ring_dt_ensemble"])


@pytest.mark.gpu
@pytest.mark.parametrize("run", GOLDEN_CPP)
def test_driver_reproduces_golden_runs(driver, golden, tmp_path, run):
    g = golden[run]
    out = tmp_path / run
    r = subprocess.run([driver, g["script"], *g["args"], "--o", str(out)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    rows, log = read_trajectory_file(out)
    ref = np.array(g["rows"])
    assert rows.shape == ref.shape
    assert np.allclose(rows, ref)
    text = "\n".join(log)
    lines = [l.rstrip("\n") for l in open(out)]
    i = lines.index("#  2. dtDid") + 1
    key = []
    while lines[i].startswith("#"):
        key.append(lines[i][2:])
        i += 1
    assert key == g["key"]
    if "ensemble_log" in g:
        for key, want in g["ensemble_log"].items():
            if key == "histogram":
                assert "Too few jumps for a histogram" in text
                continue
            m = re.search(LOG_PATTERNS[key], text)
            assert m, key
            got = float(m.group(1))
            if key == "average_overshot" and "--NDt" not in g["args"]:
                # the last interval of Dt mode is the floating-point remainder T - 10 Dt; whether
                # its step overshoots dpLimit is a last-bit tie (one per trajectory at most)
                assert abs(got - want) <= 1.0 + 1e-9, (key, got, want)
                continue
            assert np.isclose(got, want, rtol=2e-5, atol=5e-7), (key, got, want)


@pytest.mark.gpu
def test_driver_histogram_counts_every_jump(driver, engine, tmp_path):
    """With enough jumps the ensemble log carries the histogram of all jump times (the
    reference's EnsembleLogger::stream: total / 50 bins between the first and the last jump,
    plus an underflow and an overflow bin).  The same trajectories run from Python, with a
    ring large enough to keep every record, give the same histogram."""
    from cppqed_b200.evolve import _density

    args = ["--picture", "Sch", "--deltaA", "0", "--gamma", "0.5", "--deltaC", "0", "--kappa", "1", "--eta", "1.5",
            "--cutoff", "20", "--g", "2", "--evol", "ensemble", "--nTraj", "64", "--dc", "0", "--Dt", "0.5",
            "--T", "4"]
    out = tmp_path / "qbitmode"
    r = subprocess.run([driver, "QbitMode_C++QED", *args, "--o", str(out)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    text = open(out).read()
    m = re.search(r"Histogram of jumps. Number of bins=(\d+)\n((?:# \S+\t\S+\n)+)", text)
    assert m, text[-2000:]
    hist = np.array([[float(x) for x in l[2:].split("\t")] for l in m.group(2).splitlines()])
    n_avg = float(re.search(LOG_PATTERNS["average_jumps"], text).group(1))

    model = engine.Model("QbitMode_C++QED", args)
    rp = model.run_pars()
    ens = engine.Ensemble(engine.System(model.desc), model.initial_state(), 64, rp.mcwf)
    assert engine.lib().cqg_ensemble_set_jump_capacity(ens._h, 1 << 14) == A.CQG_OK
    ens.run(0.5, 8)
    times = np.concatenate([ens.jumps(i, 1 << 14)[0] for i in range(64)])
    assert abs(len(times) / 64 - n_avg) <= 1e-5 * n_avg
    want = np.array(_density(list(times), len(times) // 50))
    assert int(m.group(1)) == len(want)
    assert np.allclose(hist, want, rtol=1e-5, atol=1e-6)
    assert abs(hist[:, 1].sum() - 1) < 1e-5
