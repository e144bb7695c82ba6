"""Run the reference binaries built by oracle/ref_build.py and store their outputs as golden
fixtures (.npz).

TEST INFRASTRUCTURE ONLY.  Needs a GPU (the reference is CUDA-only).  Usage on the GPU
machine, from the repository root:

    python oracle/make_golden.py [--out DIR] [case ...]

Each case runs `oracle/_ref/<case>/cuSHG <power> <waist> <temp> 1 <save_T>` (the argv of
src/cuSHG.cu:46-58) in a scratch folder, then reads its ASCII outputs:
Pump_out_{r,i}.dat and Signal_out_{r,i}.dat (NY rows of NX tab-separated values,
src/headers/Files.h:69-90) and, for thermal cases, Tfinal_<z>.dat (src/headers/Files.h:169-202).
The .npz holds pump, signal (complex128), T (float64, nz x ny x nx) when present, the
parameter set as JSON, and the wall time of the run (for temperature grids above FULL_T_MAX
voxels: the slices T_SLICES and FP64 sums over all voxels instead of T).  The default output
folder is tests/golden/.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
from oracle.golden_cases import CASES, FULL_CASES, T_SLICES  # noqa: E402

ALL_CASES = {**CASES, **FULL_CASES}
# a temperature grid above this many voxels is stored as the slices T_SLICES plus sums
FULL_T_MAX = 1 << 20


def read_matrix(path: str, ny: int, nx: int) -> np.ndarray:
    rows = []
    with open(path) as fh:
        for line in fh:
            vals = [v for v in line.strip().split("\t") if v != ""]
            if vals:
                rows.append([float(v) for v in vals])
    a = np.asarray(rows, dtype=np.float64)
    if a.shape != (ny, nx):
        raise RuntimeError(f"{path}: shape {a.shape}, expected {(ny, nx)}")
    return a


def run_case(name: str, out_dir: str, timeout: float) -> dict:
    case = ALL_CASES[name]
    p = case["params"]
    exe = os.path.join(HERE, "_ref", name, "cuSHG")
    if not os.path.exists(exe):
        raise FileNotFoundError(exe)
    thermal = bool(p["thermal"])
    argv = [exe, repr(p["power"]), repr(p["waist"]), repr(p["temp"]), "1", "1" if thermal else "0"]
    with tempfile.TemporaryDirectory() as wd:
        t0 = time.perf_counter()
        r = subprocess.run(argv, cwd=wd, capture_output=True, text=True, timeout=timeout)
        wall = time.perf_counter() - t0
        if r.returncode != 0:
            raise RuntimeError(f"{name}: exit {r.returncode}\n{r.stdout[-2000:]}\n{r.stderr[-2000:]}")
        ny, nx, nz = p["ny"], p["nx"], p["nz"]
        pump = read_matrix(os.path.join(wd, "Pump_out_r.dat"), ny, nx) + 1j * read_matrix(os.path.join(wd, "Pump_out_i.dat"), ny, nx)
        sig = read_matrix(os.path.join(wd, "Signal_out_r.dat"), ny, nx) + 1j * read_matrix(os.path.join(wd, "Signal_out_i.dat"), ny, nx)
        arrays = {"pump": pump.astype(np.complex128), "signal": sig.astype(np.complex128)}
        if thermal:
            T = np.stack([read_matrix(os.path.join(wd, f"Tfinal_{z}.dat"), ny, nx) for z in range(nz)])
            if T.size <= FULL_T_MAX:
                arrays["T"] = T
            else:
                zs = [z for z in T_SLICES if z < nz]
                arrays["T_z"] = np.asarray(zs, dtype=np.int64)
                arrays["T_slices"] = T[zs]
                arrays["T_sum"] = np.asarray(float(np.sum(T, dtype=np.float64)))
                arrays["T_sumsq"] = np.asarray(float(np.sum(T * T, dtype=np.float64)))
                arrays["T_min"] = np.asarray(float(T.min()))
                arrays["T_max"] = np.asarray(float(T.max()))
        # iteration counts printed by the reference's thermal loop (Solver.h:356)
        sweeps = [int(tok.split()[0]) for tok in r.stdout.replace("\r", "\n").split("\n")
                  if tok.strip().endswith("iterations -> steady-state.")]
    meta = {"case": name, "precision": case["precision"], "params": p, "wall_s": wall,
            "jacobi_sweeps": sweeps, "argv": argv[1:]}
    os.makedirs(out_dir, exist_ok=True)
    np.savez_compressed(os.path.join(out_dir, name + ".npz"), meta=json.dumps(meta), **arrays)
    return meta


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(os.path.dirname(HERE), "tests", "golden"))
    ap.add_argument("--timeout", type=float, default=600.0)
    ap.add_argument("cases", nargs="*")
    a = ap.parse_args()
    names = a.cases or list(ALL_CASES)
    rc = 0
    for n in names:
        try:
            meta = run_case(n, a.out, a.timeout)
            print(json.dumps({k: meta[k] for k in ("case", "wall_s", "jacobi_sweeps")}))
        except Exception as e:  # report and continue with the other cases
            print(f"FAILED {n}: {e}")
            rc = 1
    return rc


if __name__ == "__main__":
    sys.exit(main())
