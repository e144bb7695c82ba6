"""Parameter set of the SHG solver: the ctypes mirror of ``shg_params`` / ``shg_stats``
(include/shg.h) and builders for the standard workloads.

The reference keeps these values as compile-time constants and ``argv``:
grid in src/cuSHG.cu:11-13, crystal and beam in src/headers/Crystal.h:19-52, and the
``Solver::run`` arguments in src/cuSHG.cu:46-58.  Here they are one runtime struct.
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass

import numpy as np

# status codes (include/shg.h)
SHG_OK = 0
SHG_ERR_INVALID = 1
SHG_ERR_UNSUPPORTED = 2
SHG_ERR_CUDA = 3
SHG_ERR_NOMEM = 4
SHG_ERR_NOT_CONVERGED = 5
SHG_ERR_NO_DEVICE = 6
SHG_ERR_NONFINITE = 7

SHG_BOUNDARY_TOP_OPEN = 0
SHG_BOUNDARY_OVEN_SURROUNDED = 1
SHG_CONV_REFERENCE = 0
SHG_CONV_MAXABS = 1
SHG_CONV_FIXED = 2
SHG_HEAT_JACOBI = 0
SHG_HEAT_DIRECT = 1
SHG_MARCH_AUTO = 0
SHG_MARCH_FUSED = 1
SHG_MARCH_MULTIPASS = 2
SHG_CRYSTAL_MGO_SPPLT = 0
SHG_CRYSTAL_MGO_PPLN = 1

# physical constants of src/headers/Crystal.h:19-21 (µm, ps, W, V)
C_UM_PS = 299792458 * 1e6 / 1e12
EPS0 = 8.8541878128e-12 * 1e12 / 1e6


class ShgParams(ctypes.Structure):
    """``shg_params`` of include/shg.h, field for field."""

    _fields_ = [
        ("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("lx", ctypes.c_double), ("ly", ctypes.c_double), ("lz", ctypes.c_double),
        ("lambda_p", ctypes.c_double), ("deff", ctypes.c_double), ("period", ctypes.c_double),
        ("alpha_p", ctypes.c_double), ("alpha_s", ctypes.c_double), ("beta_s", ctypes.c_double),
        ("rho_p", ctypes.c_double), ("rho_s", ctypes.c_double),
        ("kappa", ctypes.c_double), ("h_conv", ctypes.c_double),
        ("power", ctypes.c_double), ("waist", ctypes.c_double), ("focus", ctypes.c_double),
        ("temp", ctypes.c_double), ("t_inf", ctypes.c_double), ("t_peltier", ctypes.c_double),
        ("thermal", ctypes.c_int32), ("boundary", ctypes.c_int32),
        ("max_outer", ctypes.c_int32), ("check_every", ctypes.c_int32),
        ("conv_rule", ctypes.c_int32), ("crystal", ctypes.c_int32),
        ("jacobi_tol", ctypes.c_double), ("max_sweeps", ctypes.c_int64),
        ("jacobi_block", ctypes.c_int32), ("march", ctypes.c_int32),
        ("heat_solver", ctypes.c_int32), ("waist_y", ctypes.c_double),
        ("fp32_guard", ctypes.c_double),
    ]

    def copy(self) -> "ShgParams":
        q = ShgParams()
        ctypes.pointer(q)[0] = self
        return q

    def replace(self, **kw) -> "ShgParams":
        q = self.copy()
        for k, v in kw.items():
            if not hasattr(q, k):
                raise AttributeError(k)
            setattr(q, k, v)
        return q

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}

    @property
    def points(self) -> int:
        return int(self.nx) * int(self.ny)

    @property
    def real_dtype(self):
        return np.float64 if self.precision == 64 else np.float32

    @property
    def complex_dtype(self):
        return np.complex128 if self.precision == 64 else np.complex64

    def __repr__(self) -> str:  # pragma: no cover - debugging aid
        return "ShgParams(" + ", ".join(f"{k}={v!r}" for k, v in self.as_dict().items()) + ")"


class ShgStats(ctypes.Structure):
    """``shg_stats`` of include/shg.h."""

    _fields_ = [
        ("sh_power", ctypes.c_double), ("pump_power", ctypes.c_double),
        ("jacobi_sweeps", ctypes.c_int64), ("outer_iterations", ctypes.c_int32),
        ("steps", ctypes.c_int32), ("last_residual", ctypes.c_double),
        ("device_ms", ctypes.c_double), ("jacobi_ms", ctypes.c_double), ("optics_ms", ctypes.c_double),
    ]


def sellmeier(lam_um: float, temp_c: float, crystal: int = SHG_CRYSTAL_MGO_SPPLT) -> float:
    """Extraordinary index of MgO:sPPLT (Bruner et al.), src/headers/Crystal.h:54-70, or with
    ``crystal = SHG_CRYSTAL_MGO_PPLN`` of 5 mol% MgO:PPLN (Gayer et al., Appl. Phys. B 91, 343
    (2008))."""
    if crystal == SHG_CRYSTAL_MGO_PPLN:
        f = (temp_c - 24.5) * (temp_c + 570.82)
        l2 = lam_um * lam_um
        p = 0.2020 + 6.113e-8 * f
        return math.sqrt(5.756 + 2.860e-6 * f + (0.0983 + 4.700e-8 * f) / (l2 - p * p)
                         + (189.32 + 1.516e-4 * f) / (l2 - 12.52 * 12.52) - 1.32e-2 * l2)
    A, B, C, D = 4.502483, 0.007294, 0.185087, -0.02357
    E, F, G, H = 0.073423, 0.199595, 0.001, 7.99724
    tk = temp_c + 273.15
    b = 3.483933e-8 * tk * tk
    c = 1.607839e-8 * tk * tk
    l2 = lam_um * lam_um
    return math.sqrt(A + (B + b) / (l2 - (C + c) ** 2) + E / (l2 - F * F) + G / (l2 - H * H) + D * l2)


def qpm_period(temp_c: float, lambda_p: float = 1.064, crystal: int = SHG_CRYSTAL_MGO_SPPLT) -> float:
    """Grating period that zeroes Δk of src/headers/PhaseMatching.h:47-85 at ``temp_c``,
    including the grating's thermal expansion (sPPLT α = 2.2e-6, β = -5.9e-9; MgO:PPLN
    α = 1.54e-5, β = 5.3e-9)."""
    ls = 0.5 * lambda_p
    d = temp_c - 25.0
    a, b = (1.54e-5, 5.3e-9) if crystal == SHG_CRYSTAL_MGO_PPLN else (2.2e-6, -5.9e-9)
    expansion = 1.0 + a * d + b * d * d
    return 1.0 / ((sellmeier(ls, temp_c, crystal) / ls - 2.0 * sellmeier(lambda_p, temp_c, crystal) / lambda_p)
                  * expansion)


def reference_defaults() -> ShgParams:
    """The reference's own compile-time configuration: src/cuSHG.cu:11-13 and 46-53,
    src/headers/Crystal.h:19-52, with the argv of src/cuSHG.sh:43-45 (30 W, 29 µm,
    55.66 °C).  Identical to shg_default_params() of the C ABI."""
    p = ShgParams()
    p.nx, p.ny, p.nz, p.precision = 128, 128, 100, 32
    p.lx, p.ly, p.lz = 2000.0, 1000.0, 30000.0
    p.lambda_p, p.deff, p.period = 1.064, 11.00e-6, 7.97
    p.alpha_p, p.alpha_s, p.beta_s = 0.17e-6, 1.57e-6, 5e-5
    p.rho_p = p.rho_s = 0.0
    p.kappa, p.h_conv = 8.4e-6, 10e-12
    p.power, p.waist, p.focus = 30.0, 29.0, 0.5 * 30000.0
    p.temp, p.t_inf, p.t_peltier = 55.66, 25.0, 55.66
    p.thermal, p.boundary = 0, SHG_BOUNDARY_TOP_OPEN
    p.max_outer, p.check_every = 20, 5000
    p.conv_rule, p.crystal = SHG_CONV_REFERENCE, 0
    p.jacobi_tol, p.max_sweeps = 0.0, 0
    return p


# ---------------------------------------------------------------------------------
# Standard workloads.  Units: µm, W, °C.  Absorption: α_ω = 0.002 cm⁻¹, α_2ω = 0.04 cm⁻¹,
# β = 1e-11 m/W = 1e-5 µm/W; d_eff = 10 pm/V = 1e-5 µm/V; the window is 12·w0 square.

ALPHA_P = 0.002e-4
ALPHA_S = 0.04e-4
BETA_S = 1e-5
DEFF = 10e-6
QPM_TEMP = 27.0


def workload(n: int, nz: int, lz: float, power: float, waist: float, focus: float,
             temp: float, precision: int = 64, thermal: int = 0) -> ShgParams:
    p = reference_defaults()
    p.nx = p.ny = int(n)
    p.nz = int(nz)
    p.precision = int(precision)
    p.lx = p.ly = 12.0 * waist
    p.lz = float(lz)
    p.deff = DEFF
    p.period = qpm_period(QPM_TEMP)
    p.alpha_p, p.alpha_s, p.beta_s = ALPHA_P, ALPHA_S, BETA_S
    p.power, p.waist, p.focus = float(power), float(waist), float(focus)
    p.temp = p.t_peltier = float(temp)
    p.t_inf = 25.0
    p.thermal = int(thermal)
    return p


def config_plain_64() -> ShgParams:
    """Plain FP64 run on a 64x64 grid, nz = 100: 10 mm crystal, 5 W, w0 = 30 µm focused
    at the centre, QPM at 27 °C, SH starting at zero."""
    return workload(64, 100, 10000.0, 5.0, 30.0, 5000.0, QPM_TEMP, precision=64)


def config_thermal_128() -> ShgParams:
    """Thermal FP64 run: 128x128 optical grid, nz = 200, 20 mm crystal, 20 W, w0 = 40 µm,
    128x128x200 temperature grid with the oven at 40 °C, κ = 8.4 W/(m K), Jacobi to
    max|ΔT| < 1e-6 K inside 5 outer optical-thermal iterations."""
    p = workload(128, 200, 20000.0, 20.0, 40.0, 10000.0, 40.0, precision=64, thermal=1)
    p.max_outer = 5
    p.conv_rule = SHG_CONV_MAXABS
    p.jacobi_tol = 1e-6
    p.check_every = 1000
    return p


def config_sweep(count: int = 256, seed: int = 0, precision: int = 32) -> list[ShgParams]:
    """Batched parameter sweep: `count` instances from `seed` with grid side in
    {64, 128, 192, 256}, nz in [100, 400], P log-uniform in [1, 50] W, w0 uniform in
    [15, 60] µm, focus uniform over the crystal, oven temperature uniform in [20, 80] °C
    and L in {10, 20} mm."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = int(rng.choice([64, 128, 192, 256]))
        nz = int(rng.integers(100, 401))
        power = float(math.exp(rng.uniform(math.log(1.0), math.log(50.0))))
        waist = float(rng.uniform(15.0, 60.0))
        lz = float(rng.choice([10000.0, 20000.0]))
        focus = float(rng.uniform(0.0, lz))
        temp = float(rng.uniform(20.0, 80.0))
        out.append(workload(n, nz, lz, power, waist, focus, temp, precision=precision))
    return out


def config_adjoint() -> ShgParams:
    """Adjoint workload: 256x256, nz = 400, 20 mm, 30 W, w0 = 35 µm, focus at 0.4 L, 30 °C."""
    return workload(256, 400, 20000.0, 30.0, 35.0, 8000.0, 30.0, precision=32)


def config_thermal_512(count: int = 8) -> list[ShgParams]:
    """Large thermal batch: 512x512, nz = 1000, FP32 fields, 50 W, w0 = 50 µm, 20 mm,
    ovens evenly spaced over 30-65 °C."""
    temps = np.linspace(30.0, 65.0, count)
    out = []
    for t in temps:
        p = workload(512, 1000, 20000.0, 50.0, 50.0, 10000.0, float(t), precision=32, thermal=1)
        p.max_outer = 5
        p.conv_rule = SHG_CONV_MAXABS
        p.jacobi_tol = 1e-6
        p.check_every = 1000
        out.append(p)
    return out


@dataclass
class Result:
    """Fields and report of one solve."""

    pump: np.ndarray
    signal: np.ndarray
    stats: ShgStats
    temperature: np.ndarray | None = None

    @property
    def sh_power(self) -> float:
        return float(self.stats.sh_power)


def sh_power_of(p: ShgParams, signal: np.ndarray, temp: float | None = None) -> float:
    """SH power Σ ½ ε0 c n_s |S|² dx dy (n_s at ``temp``, default p.temp), summed in double."""
    t = p.temp if temp is None else temp
    ns = sellmeier(0.5 * p.lambda_p, t, p.crystal)
    dx = p.lx / (p.nx - 1)
    dy = p.ly / (p.ny - 1)
    return float(0.5 * EPS0 * C_UM_PS * ns * np.sum(np.abs(signal.astype(np.complex128)) ** 2) * dx * dy)
