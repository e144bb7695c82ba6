"""cushg_b200 — B200-native (sm_100a) solver for the focused-beam SHG hot path of
alfredos84/cuSHG: the split-step Fourier march of the pump and second-harmonic fields and
the 3D Jacobi heat solve, behind the C ABI of include/shg.h (libshg_b200.so)."""
from .params import (ShgParams, ShgStats, Result, reference_defaults, workload, config_plain_64,  # noqa: F401
                     config_thermal_128, config_sweep, config_adjoint, config_thermal_512, qpm_period,
                     sellmeier, sh_power_of)

__all__ = ["ShgParams", "ShgStats", "Result", "reference_defaults", "workload", "config_plain_64",
           "config_thermal_128", "config_sweep", "config_adjoint", "config_thermal_512", "qpm_period",
           "sellmeier", "sh_power_of"]
