#!/usr/bin/env python3
"""Extract the golden vectors used by the parity tests from the reference's own test data.

Run in a container that has the reference checked out (--reference DIR; default
$NSE2D_REFERENCE_DIR, else the directory "reference" beside this repository). Writes
tests/golden/reference_cases.json: for every case of the reference test suite
(tests/run_tests.py:72-111 of the reference) its command line, the header of its
diagnostics.csv and its first rows (the t = 0 row is a deterministic function of the
initial condition; the early rows are deterministic up to round-off), plus the reference's
tests/reference/reference.json values and the relative tolerances REF_TOL
(tests/run_tests.py:342-345). No reference source code is copied.
"""
import argparse
import json
import os

ap = argparse.ArgumentParser()
_REPO = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
ap.add_argument("--reference", default=os.environ.get("NSE2D_REFERENCE_DIR")
                or os.path.join(os.path.dirname(_REPO), "reference"))
ap.add_argument("--rows", type=int, default=6)
args = ap.parse_args()

out_dir = os.path.join(args.reference, "tests", "reference", "output")
cases = {}
for case in sorted(os.listdir(out_dir)):
    d = os.path.join(out_dir, case)
    cmd = open(os.path.join(d, "command.txt")).read().split()
    with open(os.path.join(d, "diagnostics.csv")) as f:
        lines = [ln.strip() for ln in f if ln.strip()]
    header = lines[0].split(",")
    rows = [[float(x) for x in ln.split(",")] for ln in lines[1:1 + args.rows]]
    cases[case] = {"exe": cmd[0], "args": cmd[1:cmd.index("--outdir")], "header": header, "rows": rows,
                   "n_rows_total": len(lines) - 1}
ref = json.load(open(os.path.join(args.reference, "tests", "reference", "reference.json")))
doc = {"source": "xupingxie/nse2d-channel-gpu tests/reference (A100, CUDA 13.2)",
       "ref_tol": {"eigenmode_space": 0.02, "eigenmode_time": 0.05, "poiseuille": 0.05, "mms": 0.02,
                   "conservation": 0.5, "channel": 1e-4},
       "ref_abs_floor": 1e-13, "reference_json": ref, "cases": cases}
path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_cases.json")
with open(path, "w") as f:
    json.dump(doc, f, indent=1)
print("wrote", path, len(cases), "cases")
