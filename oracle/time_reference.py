"""Time the reference program against this library's command-line drop-in, process to
process, on the same inputs.

TEST INFRASTRUCTURE ONLY (measurement).  Needs a GPU.  For every case it runs the reference
binary built by oracle/ref_build.py (oracle/_ref/<case>/cuSHG with the reference's argv) and
cushg_b200/cushg with the same parameters, each in a scratch folder writing the same .dat
files, and reports both wall times (median of --repeat runs) as JSON lines.

    python oracle/time_reference.py [--repeat 3] [case ...]
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)
from oracle.golden_cases import CASES, TIMING_CASES, params_of  # noqa: E402

CLI = os.path.join(ROOT, "cushg_b200", "cushg")


def cli_argv(p):
    a = [CLI, repr(p.power), repr(p.waist), repr(p.temp), "1", "0", "--nx", str(p.nx), "--nz", str(p.nz),
         "--lx", repr(p.lx), "--ly", repr(p.ly), "--lz", repr(p.lz), "--focus", repr(p.focus),
         "--t-inf", repr(p.t_inf), "--deff", repr(p.deff), "--period", repr(p.period), "--alpha-p", repr(p.alpha_p),
         "--alpha-s", repr(p.alpha_s), "--beta-s", repr(p.beta_s), "--rho-p", repr(p.rho_p), "--rho-s", repr(p.rho_s),
         "--kappa", repr(p.kappa), "--h-conv", repr(p.h_conv), "--precision", str(p.precision)]
    if p.thermal:
        a += ["--thermal", "--max-outer", str(p.max_outer), "--check-every", str(p.check_every)]
        if p.boundary == 1:
            a += ["--boundary", "oven-surrounded"]
    return a


def wall(argv, repeat):
    ts = []
    for _ in range(repeat):
        with tempfile.TemporaryDirectory() as wd:
            t0 = time.perf_counter()
            r = subprocess.run(argv, cwd=wd, capture_output=True, text=True, timeout=3600)
            ts.append(time.perf_counter() - t0)
            if r.returncode != 0:
                raise RuntimeError(f"{argv[0]} failed: {r.stderr[-500:]}")
    return statistics.median(ts)


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--repeat", type=int, default=3)
    ap.add_argument("cases", nargs="*")
    a = ap.parse_args()
    names = a.cases or [n for n in {**CASES, **TIMING_CASES} if not CASES.get(n, {}).get("params", {}).get("thermal")]
    for n in names:
        p = params_of(n)
        ref = [os.path.join(HERE, "_ref", n, "cuSHG"), repr(p.power), repr(p.waist), repr(p.temp), "1",
               "1" if p.thermal else "0"]
        t_ref = wall(ref, a.repeat)
        t_ours = wall(cli_argv(p), a.repeat)
        print(json.dumps({"case": n, "grid": [p.nx, p.ny, p.nz], "precision": p.precision, "thermal": p.thermal,
                          "reference_wall_s": t_ref, "ours_wall_s": t_ours, "speedup": t_ref / t_ours}), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
