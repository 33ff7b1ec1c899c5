"""Writes master_equation_runs.json: the oracle's FP64 master-equation evolution
(quantumtrajectory::Master, Master.h:153-208, as restated in oracle/oracle.cpp) of the
workloads whose ensemble averages the bench states an error against.

Each entry holds the script, its arguments, the output interval Dt, the end time T and the
streamed rows (t, dtDid, processed averages) of `--evol master`.  A CPU test recomputes them
with the oracle and requires the same numbers, so the fixture cannot drift from the oracle.

usage: python tests/golden/make_master_fixtures.py
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

# name: (script, args, T, Dt)
RUNS = {
    "qbitmode_jc_2x40": ("QbitMode_C++QED",
                         ["--picture", "Sch", "--deltaA", "0", "--gamma", "0.5", "--deltaC", "0", "--kappa", "1",
                          "--eta", "1.5", "--cutoff", "40", "--g", "2"], 20.0, 1.0),
}


def master_rows(script, args, T, Dt):
    import cppqed_b200 as cqg
    from cppqed_b200 import _abi as A
    from tests.oracle_lib import Oracle

    model = cqg.Model(script, args)
    rp = model.run_pars()
    rp.evol = A.EVOL_MASTER
    rp.dc = 0
    rp.T = T
    rp.Dt = Dt
    rp.NDt = 0
    return Oracle().run(model, rp), model.key()


def main():
    out = {}
    for name, (script, args, T, Dt) in RUNS.items():
        rows, key = master_rows(script, args, T, Dt)
        out[name] = {"script": script, "args": args, "T": T, "Dt": Dt, "key": key, "rows": rows.tolist()}
    dst = os.path.join(HERE, "master_equation_runs.json")
    json.dump(out, open(dst, "w"), indent=0)
    print("wrote", dst, len(out), "runs")


if __name__ == "__main__":
    main()
