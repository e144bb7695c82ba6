"""Build the reference program (alfredos84/cuSHG) for sm_100a, one binary per golden case.

TEST INFRASTRUCTURE ONLY.  The reference is a single-translation-unit CUDA program whose
grid, crystal and beam constants are compile-time values and which is float-only.  To use
it as the parity oracle this recipe copies its sources into oracle/_ref/<case>/ (a
git-ignored build folder), applies the patch set below, and compiles it with nvcc
directly (the reference ships no build system beyond one nvcc line in src/cuSHG.sh:22-27).

Patch set (every pattern must match, or the build stops):
  * precision 64: real_t = double, complex_t = cufftDoubleComplex (src/cuSHG.cu:7-8),
    make_cuComplex / make_cuFloatComplex -> make_cuDoubleComplex, CUFFT_C2C -> CUFFT_Z2Z,
    cufftExecC2C -> cufftExecZ2Z, and the float-only math calls (cosf sinf expf sqrtf powf
    tanf) -> their double forms, so nothing is silently truncated to float;
  * grid NX, NY, NZ (src/cuSHG.cu:11-13) and crystal constants (src/headers/Crystal.h:31-48);
  * focal point (src/cuSHG.cu:48, hard-wired to 0.5*LZ there);
  * SH initial field = 0 instead of clock-seeded noise (src/headers/Efields.h:221-226);
  * outer optical-thermal iteration count (src/headers/Solver.h:325);
  * temperature dump at 20 significant digits (src/headers/Files.h:179).

Run where the reference checkout and nvcc are (no GPU needed):
    python oracle/ref_build.py [--reference DIR] [case ...]    # default: all cases
DIR is the reference checkout (the folder holding src/cuSHG.cu).  Without --reference it is
taken from the environment variable CUSHG_REFERENCE, else from a folder named `reference`
beside this repository.
The binaries travel to the GPU machine with the repository snapshot; make_golden.py runs
them there.
"""
from __future__ import annotations

import json
import os
import re
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def reference_src(path: str | None = None) -> str:
    """The reference's src/ folder: `path`, else $CUSHG_REFERENCE, else ../reference beside
    the repository."""
    root = path or os.environ.get("CUSHG_REFERENCE") or os.path.join(os.path.dirname(os.path.dirname(HERE)),
                                                                      "reference")
    return os.path.join(root, "src")

OUT = os.path.join(HERE, "_ref")

sys.path.insert(0, os.path.dirname(HERE))
from oracle.golden_cases import CASES, FULL_CASES, TIMING_CASES  # noqa: E402


def _sub(text: str, pattern: str, repl: str, count_expected: int | None = None, flags=0) -> str:
    new, n = re.subn(pattern, repl, text, flags=flags)
    if n == 0 or (count_expected is not None and n != count_expected):
        raise RuntimeError(f"patch pattern {pattern!r} matched {n} times")
    return new


def _num(v: float) -> str:
    return repr(float(v))


def patch_tree(dst: str, case: dict) -> None:
    p = case["params"]
    fp64 = case["precision"] == 64
    main = os.path.join(dst, "cuSHG.cu")
    hdr = os.path.join(dst, "headers")

    s = open(main).read()
    if fp64:
        s = _sub(s, r"using real_t = float;", "using real_t = double;")
        s = _sub(s, r"using complex_t = cufftComplex;", "using complex_t = cufftDoubleComplex;")
    for name, val in (("NX", p["nx"]), ("NY", p["ny"]), ("NZ", p["nz"])):
        s = _sub(s, r"(__constant__ const uint\s+" + name + r"\s*=\s*)\d+;", r"\g<1>" + str(int(val)) + ";")
    s = _sub(s, r"real_t focalpoint\s*=\s*0\.5\*LZ;", "real_t focalpoint = " + _num(p["focus"]) + ";")
    s = _sub(s, r"real_t T_inf\s*=\s*25;", "real_t T_inf = " + _num(p["t_inf"]) + ";")
    open(main, "w").write(s)

    f = os.path.join(hdr, "Crystal.h")
    s = open(f).read()
    consts = {
        "LX": p["lx"], "LY": p["ly"], "LZ": p["lz"], "deff": p["deff"], "Lambda": p["period"],
        "alpha_crp": p["alpha_p"], "alpha_crs": p["alpha_s"], "beta_crs": p["beta_s"],
        "rhop": p["rho_p"], "rhos": p["rho_s"], "thermal_cond": p["kappa"], "heat_trf_coeff": p["h_conv"],
    }
    for name, val in consts.items():
        s = _sub(s, r"(__constant__ const real_t\s+" + name + r"\s*=\s*)[^;]+;", r"\g<1>" + _num(val) + ";", 1)
    s = _sub(s, r"(__constant__ const real_t\s+lp\s*=\s*)[^;]+;", r"\g<1>" + _num(p["lambda_p"]) + ";", 1)
    open(f, "w").write(s)

    f = os.path.join(hdr, "Efields.h")
    s = open(f).read()
    s = _sub(s, r"noiseGeneratorGPU \( this->Signal \);", "CHECK(cudaMemset(this->Signal, 0, nBytes2Dc));", 1)
    if fp64:
        s = _sub(s, r"make_cuComplex\(", "make_cuDoubleComplex(")
        for fn in ("sqrtf", "powf", "tanf"):
            s = _sub(s, r"\b" + fn + r"\(", fn[:-1] + "(")
    open(f, "w").write(s)

    f = os.path.join(hdr, "Solver.h")
    s = open(f).read()
    s = _sub(s, r"num_of_iter = 20;", "num_of_iter = " + str(int(p["max_outer"])) + ";", 1)
    if case.get("oven_surrounded"):
        s = _sub(s, r"T->setBottomOvens\( Tpeltier\);", "T->setOvenSurrounded( Tpeltier);", 1)
    if fp64:
        s = _sub(s, r"make_cuComplex\(", "make_cuDoubleComplex(")
        s = _sub(s, r"CUFFT_C2C", "CUFFT_Z2Z")
        s = _sub(s, r"cufftExecC2C", "cufftExecZ2Z")
    open(f, "w").write(s)

    if case.get("oven_surrounded"):
        f = os.path.join(hdr, "Tfield.h")
        s = open(f).read()
        s = _sub(s, r"kernelHeatEquationTopOpen<<<", "kernelHeatEquationOvenSurrounded<<<", 1)
        open(f, "w").write(s)

    f = os.path.join(hdr, "Operators.h")
    s = open(f).read()
    if fp64:
        for fn in ("cosf", "sinf", "expf", "sqrtf"):
            s = _sub(s, r"\b" + fn + r"\(", fn[:-1] + "(")
        s = _sub(s, r"make_cuFloatComplex\(", "make_cuDoubleComplex(")
    open(f, "w").write(s)

    f = os.path.join(hdr, "PhaseMatching.h")
    s = open(f).read()
    if fp64:
        s = _sub(s, r"\bpowf\(", "pow(")
    open(f, "w").write(s)

    f = os.path.join(hdr, "Tfield.h")
    s = open(f).read()
    if fp64:
        s = _sub(s, r"\bpowf\(", "pow(")
    open(f, "w").write(s)

    f = os.path.join(hdr, "Files.h")
    s = open(f).read()
    s = _sub(s, r"myfile << Tensor\[IDX\(ix,iy,iz\)\] << \"\\t\";",
             'myfile << std::setprecision(20) << Tensor[IDX(ix,iy,iz)] << "\\t";', 1)
    open(f, "w").write(s)


def build_case(name: str, case: dict, nvcc: str = "nvcc", src: str | None = None) -> str:
    src = src or reference_src()
    dst = os.path.join(OUT, name, "src")
    if os.path.isdir(os.path.join(OUT, name)):
        shutil.rmtree(os.path.join(OUT, name))
    shutil.copytree(src, dst)
    patch_tree(dst, case)
    exe = os.path.join(OUT, name, "cuSHG")
    cmd = [nvcc, "-O3", "-gencode", "arch=compute_100a,code=sm_100a", "cuSHG.cu", "-o", exe, "-lcufftw", "-lcufft"]
    if case["params"]["thermal"]:
        cmd.insert(1, "-DTHERMAL")
    subprocess.run(cmd, cwd=dst, check=True)
    # keep only the binary: the patched sources are an intermediate of this build
    shutil.rmtree(dst)
    with open(os.path.join(OUT, name, "case.json"), "w") as fh:
        json.dump({"name": name, **case}, fh, indent=1)
    return exe


def main(argv: list[str]) -> int:
    import argparse

    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=None, help="reference checkout (the folder holding src/cuSHG.cu)")
    ap.add_argument("cases", nargs="*")
    a = ap.parse_args(argv[1:])
    src = reference_src(a.reference)
    if not os.path.isdir(src):
        print(f"reference sources not present at {src}; nothing to build")
        return 0
    allc = {**CASES, **FULL_CASES, **TIMING_CASES}
    for n in a.cases or list(allc):
        exe = build_case(n, allc[n], src=src)
        print("built", exe)
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))
