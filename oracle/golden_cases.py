"""Golden cases: parameter sets run through the reference program (oracle/ref_build.py,
oracle/make_golden.py) to pin the CPU oracle and the CUDA path.

TEST INFRASTRUCTURE ONLY.

The reference takes its inputs as compile-time constants plus argv (src/cuSHG.cu:46-58):
argv = power, waist, oven temperature, save_only_last, save_temperature, with the
Peltier temperature equal to the oven temperature (src/cuSHG.cu:53), so every case here
has t_peltier == temp.
"""
from __future__ import annotations

import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
from cushg_b200 import params as P  # noqa: E402


def _d(p: P.ShgParams) -> dict:
    return p.as_dict()


def _plain_c1() -> P.ShgParams:
    return P.config_plain_64()


def _plain_96_walkoff() -> P.ShgParams:
    # 96 = 3 * 32 exercises a radix-3 transform; lx != ly gives dx != dy; walk-off on.
    p = P.workload(96, 40, 8000.0, 12.0, 25.0, 0.5 * 8000.0, 33.0, precision=64)
    p.lx, p.ly = 400.0, 330.0
    p.rho_p, p.rho_s = 0.004, 0.006
    p.period = 8.0
    return p


def _plain_128_offfocus() -> P.ShgParams:
    p = P.workload(128, 60, 20000.0, 30.0, 35.0, 0.5 * 20000.0, 29.0, precision=64)
    return p


def _thermal_small() -> P.ShgParams:
    # small thermal grid with strong absorption so the optical-thermal coupling is visible
    p = P.workload(24, 12, 4000.0, 20.0, 25.0, 2000.0, 30.0, precision=64, thermal=1)
    p.alpha_p, p.alpha_s, p.beta_s = 2e-5, 1e-4, 1e-3
    p.max_outer = 3
    p.check_every = 5000
    p.conv_rule = P.SHG_CONV_REFERENCE
    p.jacobi_tol = 0.0
    return p


def _thermal_small_oven() -> P.ShgParams:
    p = _thermal_small()
    p.boundary = P.SHG_BOUNDARY_OVEN_SURROUNDED
    return p


def _thermal_n32() -> P.ShgParams:
    # 32 x 32 x 16 thermal case on a grid the fused kernels support (side a multiple of 16)
    p = P.workload(32, 16, 5000.0, 25.0, 28.0, 2500.0, 31.0, precision=64, thermal=1)
    p.alpha_p, p.alpha_s, p.beta_s = 2e-5, 1e-4, 1e-3
    p.max_outer = 3
    p.check_every = 5000
    p.conv_rule = P.SHG_CONV_REFERENCE
    p.jacobi_tol = 0.0
    return p


def _thermal_n32_oven() -> P.ShgParams:
    p = _thermal_n32()
    p.boundary = P.SHG_BOUNDARY_OVEN_SURROUNDED
    return p


def _plain_c1_f32() -> P.ShgParams:
    return P.config_plain_64().replace(precision=32)


CASES = {
    "plain64_c1": {"precision": 64, "params": _d(_plain_c1())},
    "plain64_n96_walkoff": {"precision": 64, "params": _d(_plain_96_walkoff())},
    "plain64_n128": {"precision": 64, "params": _d(_plain_128_offfocus())},
    "thermal64_small": {"precision": 64, "params": _d(_thermal_small())},
    "thermal64_small_oven": {"precision": 64, "params": _d(_thermal_small_oven()), "oven_surrounded": True},
    "plain32_c1": {"precision": 32, "params": _d(_plain_c1_f32())},
    "thermal64_n32": {"precision": 64, "params": _d(_thermal_n32())},
    "thermal64_n32_oven": {"precision": 64, "params": _d(_thermal_n32_oven()), "oven_surrounded": True},
}


def _thermal_c2() -> P.ShgParams:
    # the thermal workload at its stated size: 128 x 128 x 200, 20 mm, 20 W, w0 = 40 µm, oven 40 °C,
    # 5 outer iterations, under the reference's own stopping rule (the reference binary has no
    # other): residual check every 5000 sweeps against 5e-4 / TSIZE, stagnation exit
    return P.config_thermal_128().replace(conv_rule=P.SHG_CONV_REFERENCE, jacobi_tol=0.0, check_every=5000,
                                          max_outer=5)


def _plain_c4() -> P.ShgParams:
    # the gradient workload's forward at its stated size: 256 x 256, nz = 400, 20 mm, 30 W, w0 = 35 µm,
    # focus at 0.4 L, 30 °C (the reference has no per-slice poling phase: uniform grating)
    return P.config_adjoint().replace(precision=64)


# The 128 x 128 x 200 thermal and 256 x 256 x 400 plain workloads at full size, kept apart from
# CASES because the CPU oracle needs minutes for them.  The thermal run's temperature grid
# (26 MB) is too large for a fixture,
# so make_golden.py keeps the slices T_SLICES plus FP64 sums over all voxels.
FULL_CASES = {
    "thermal64_c2": {"precision": 64, "params": _d(_thermal_c2())},
    "plain64_c4": {"precision": 64, "params": _d(_plain_c4())},
}
T_SLICES = (0, 1, 50, 99, 100, 150, 198, 199)


def _timing_256(precision: int) -> P.ShgParams:
    # 256 x 256, nz = 400, 20 mm, 30 W, w0 = 35 µm, focus at 0.4 L, 30 °C
    return P.config_adjoint().replace(precision=precision)


# Reference builds used only to time the reference program against this library
# (oracle/time_reference.py); their outputs are not stored.
TIMING_CASES = {
    "time_f32_n256_nz400": {"precision": 32, "params": _d(_timing_256(32))},
    "time_f64_n256_nz400": {"precision": 64, "params": _d(_timing_256(64))},
    "time_thermal_c2": {"precision": 64, "params": _d(P.config_thermal_128().replace(
        conv_rule=P.SHG_CONV_REFERENCE, jacobi_tol=0.0, check_every=5000, max_outer=5))},
    "time_f32_n128_nz200": {"precision": 32, "params": _d(P.workload(128, 200, 20000.0, 20.0, 40.0, 10000.0, 40.0,
                                                                       precision=32))},
}


def params_of(name: str) -> P.ShgParams:
    p = P.ShgParams()
    src = {**CASES, **FULL_CASES, **TIMING_CASES}[name]
    for k, v in src["params"].items():
        setattr(p, k, v)
    return p
