"""Extracts the numeric columns of the reference's golden runs into JSON fixtures.

Reads Testing/expected/run_<name> (C++QED v2.120, written by CPPQEDscripts with the
command lines of Testing/run/testdriver.conf) and stores, per run, the command line,
the streamed rows (time, dtDid, averages), the system's lines of the header's key to the
columns, the numbers of the end-of-run ensemble log
(mcwf::EnsembleLogger::stream: average steps, dpLimit / dpTolerance overshoots with their
maxima, maximal norm deviation, average jumps) and the pcg64 engine state serialised in
the first archive of the matching .state file (the engine right after seeding).
Run once where the reference tree is available:

    python tests/golden/make_golden.py /path/to/reference
"""
import bz2
import json
import os
import re
import sys

RUNS = ["run_PTLA_CPPQED_%s_%s" % (m, e) for m in ("dc", "dt", "ndt") for e in ("single", "ensemble", "master")]
RUNS += ["run_1particle1mode_%s_%s" % (m, e) for m in ("dc", "dt", "ndt", "ndt_conf2", "ndt_conf3", "ndt_conf4")
         for e in ("single", "ensemble", "master")]
RUNS += ["run_Ring_%s_%s" % (m, e) for m in ("dc", "dt", "ndt") for e in ("single", "ensemble", "master")]


LOG_PATTERNS = {
    "average_steps": r"Average number of total steps: (\S+)",
    "average_overshot": r"On average, dpLimit overshot: (\S+) times",
    "max_overshoot": r"dpLimit overshot: \S+ times, maximal overshoot: (\S+)",
    "average_tolerance_overshot": r"On average, dpTolerance overshot: (\S+) times",
    "max_tolerance_overshoot": r"dpTolerance overshot: \S+ times, maximal overshoot: (\S+)",
    "max_norm_deviation": r"Maximal deviation of norm from 1: (\S+)",
    "average_jumps": r"Average number of total jumps: (\S+)",
}


def parse_key(path):
    """The system's part of the header's "Key to data" block: the lines after the
    trajectory's own columns (time, dtDid) up to the next empty line, without the "# "."""
    lines = [l.rstrip("\n") for l in open(path)]
    try:
        i = lines.index("#  2. dtDid") + 1
    except ValueError:
        return None
    key = []
    while i < len(lines) and lines[i].startswith("#"):
        key.append(lines[i][2:])
        i += 1
    return key


def parse(path):
    cmd, rows, log = None, [], {}
    for line in open(path):
        if line.startswith("#"):
            if cmd is None and line.strip() != "#":
                cmd = line[1:].strip()
            if rows:
                for key, pat in LOG_PATTERNS.items():
                    m = re.search(pat, line)
                    if m:
                        log[key] = float(m.group(1))
                if "Too few jumps for a histogram" in line:
                    log["histogram"] = False
            continue
        if line.strip():
            rows.append([float(x) for x in line.split()])
    return cmd, rows, log


def pcg_state(path):
    if not os.path.exists(path):
        return None
    raw = bz2.decompress(open(path, "rb").read())
    m = re.search(rb"(\d{20,}) (\d+) (\d{10,}) ", raw)
    return m.group(0).decode().strip() if m else None


def main(ref):
    exp = os.path.join(ref, "Testing", "expected")
    out = {}
    for r in RUNS:
        p = os.path.join(exp, r)
        if not os.path.exists(p):
            continue
        cmd, rows, log = parse(p)
        args = cmd.split()[1:]
        if "--o" in args:
            i = args.index("--o")
            del args[i:i + 2]
        out[r] = {"script": os.path.basename(cmd.split()[0]), "args": args, "rows": rows,
                  "pcg64_first_archive": pcg_state(p + ".state"), "key": parse_key(p)}
        if log:
            out[r]["ensemble_log"] = log
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_runs.json")
    json.dump(out, open(dst, "w"), indent=0)
    print("wrote", dst, len(out), "runs")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <path of the C++QED source tree>")
    main(sys.argv[1])
