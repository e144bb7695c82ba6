"""Python mirror of the reference's solver interface over the C ABI of libshg_b200.so.

The reference runs one parameter point per process: ``Solver::run(Power, waist, focalpoint,
Temp, T_inf, Tpeltier, save_only_last, save_temperature)`` (src/headers/Solver.h:311) with
grid and crystal constants compiled in, writing ``Pump_out`` / ``Signal_out`` .dat files.
Here :func:`run` takes the same arguments plus a runtime :class:`ShgParams`, and returns the
fields as arrays; :func:`solve_batch` runs many points in one persistent launch.

Everything goes through ``libshg_b200.so`` (include/shg.h).  There is no CPU path: if the
library or a CUDA device is missing, the calls raise.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from .params import ShgParams, ShgStats, Result, SHG_OK

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libshg_b200.so")

# every entry point declared in include/shg.h
EXPORTS = (
    "shg_default_params", "shg_check_params", "shg_steps", "shg_solve", "shg_solve_slices", "shg_solve_device",
    "shg_solve_batch_device", "shg_solve_batch_device_noalloc", "shg_grad", "shg_sh_power", "shg_last_error",
    "shg_status_string", "shg_version", "shg_heat_sweeps_device", "shg_batch_plan_create", "shg_batch_plan_launch",
    "shg_batch_plan_powers", "shg_batch_plan_destroy", "shg_autotune", "shg_grad_batch", "shg_solve_batch",
    "shg_thermal_grad", "shg_autotune_batch", "shg_autotune_reset", "shg_set_schedule",
    "shg_reserve_device_memory", "shg_fp32_error_estimate", "shg_selftest_bounded_wait",
    "shg_thermal_batch", "shg_heat_steady_device", "shg_heat_operator_modes",
)


class ShgThermalGradResult(ctypes.Structure):
    """``shg_thermal_grad_result`` of include/shg.h."""
    _fields_ = [("sh_power", ctypes.c_double), ("d_temp", ctypes.c_double),
                ("sh_power_tangent_march", ctypes.c_double), ("device_ms", ctypes.c_double),
                ("stats", ShgStats), ("reserved", ctypes.c_double * 4)]


class ShgTuneResult(ctypes.Structure):
    """``shg_tune_result`` of include/shg.h."""
    _fields_ = [("precision", ctypes.c_int32), ("n", ctypes.c_int32), ("cluster", ctypes.c_int32),
                ("threads", ctypes.c_int32), ("candidates", ctypes.c_int32), ("reserved", ctypes.c_int32),
                ("pt_steps_per_s", ctypes.c_double), ("default_pt_steps_per_s", ctypes.c_double)]


class ShgGradResult(ctypes.Structure):
    """``shg_grad_result`` of include/shg.h."""

    _fields_ = [
        ("sh_power", ctypes.c_double), ("d_waist", ctypes.c_double), ("d_focus", ctypes.c_double),
        ("d_temp", ctypes.c_double), ("d_poling", ctypes.POINTER(ctypes.c_double)), ("device_ms", ctypes.c_double),
        ("checkpoint_every", ctypes.c_int32), ("steps", ctypes.c_int32), ("reserved", ctypes.c_double * 4),
    ]


class ShgError(RuntimeError):
    """A non-zero shg_status from the library."""

    def __init__(self, status: int, message: str):
        super().__init__(f"shg status {status}: {message}")
        self.status = status


_lib = None


def lib() -> ctypes.CDLL:
    """Load libshg_b200.so (built by ``python -m cushg_b200.build``)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m cushg_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.POINTER(ShgParams)
        vp = ctypes.c_void_p
        L.shg_default_params.argtypes = [P]
        L.shg_default_params.restype = None
        L.shg_check_params.argtypes = [P]
        L.shg_check_params.restype = ctypes.c_int
        L.shg_thermal_batch.argtypes = [P, ctypes.c_int32, ctypes.POINTER(vp), ctypes.POINTER(vp), ctypes.POINTER(vp),
                                        ctypes.POINTER(ShgStats), ctypes.POINTER(ctypes.c_double), vp]
        L.shg_thermal_batch.restype = ctypes.c_int
        L.shg_selftest_bounded_wait.argtypes = [ctypes.c_int32, ctypes.c_double, ctypes.c_int32]
        L.shg_selftest_bounded_wait.restype = ctypes.c_int
        L.shg_fp32_error_estimate.argtypes = [P]
        L.shg_fp32_error_estimate.restype = ctypes.c_double
        L.shg_steps.argtypes = [P]
        L.shg_steps.restype = ctypes.c_int32
        L.shg_solve.argtypes = [P, vp, vp, vp, vp, ctypes.POINTER(ShgStats)]
        L.shg_solve.restype = ctypes.c_int
        L.shg_solve_slices.argtypes = [P, vp, vp, vp, vp, ctypes.POINTER(ShgStats)]
        L.shg_solve_slices.restype = ctypes.c_int
        L.shg_solve_device.argtypes = [P, vp, vp, vp, vp, ctypes.POINTER(ShgStats), vp]
        L.shg_solve_device.restype = ctypes.c_int
        L.shg_solve_batch_device.argtypes = [P, ctypes.c_int32, ctypes.POINTER(vp), ctypes.POINTER(vp),
                                             ctypes.POINTER(ctypes.c_double), vp]
        L.shg_solve_batch_device.restype = ctypes.c_int
        L.shg_solve_batch.argtypes = [P, ctypes.c_int32, ctypes.POINTER(vp), ctypes.POINTER(vp),
                                      ctypes.POINTER(ctypes.c_double)]
        L.shg_solve_batch.restype = ctypes.c_int
        L.shg_solve_batch_device_noalloc.argtypes = L.shg_solve_batch_device.argtypes
        L.shg_solve_batch_device_noalloc.restype = ctypes.c_int
        L.shg_grad.argtypes = [P, ctypes.POINTER(ctypes.c_double), ctypes.c_int32, ctypes.POINTER(ShgGradResult)]
        L.shg_grad.restype = ctypes.c_int
        L.shg_grad_batch.argtypes = [P, ctypes.c_int32, ctypes.POINTER(ctypes.POINTER(ctypes.c_double)),
                                     ctypes.c_int32, ctypes.POINTER(ShgGradResult)]
        L.shg_grad_batch.restype = ctypes.c_int
        L.shg_sh_power.argtypes = [P, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
        L.shg_sh_power.restype = ctypes.c_int
        L.shg_heat_sweeps_device.argtypes = [P, vp, vp, ctypes.c_int64, vp]
        L.shg_heat_sweeps_device.restype = ctypes.c_int
        L.shg_heat_steady_device.argtypes = [P, vp, vp, ctypes.POINTER(ctypes.c_double), vp]
        L.shg_heat_steady_device.restype = ctypes.c_int
        L.shg_heat_operator_modes.argtypes = [ctypes.c_int32, ctypes.c_double, ctypes.c_int32, ctypes.c_int32,
                                              ctypes.c_double] + [ctypes.POINTER(ctypes.c_double)] * 3
        L.shg_heat_operator_modes.restype = ctypes.c_int
        L.shg_batch_plan_create.argtypes = [P, ctypes.c_int32, ctypes.POINTER(vp), ctypes.POINTER(vp),
                                            ctypes.POINTER(vp)]
        L.shg_batch_plan_create.restype = ctypes.c_int
        L.shg_batch_plan_launch.argtypes = [vp, vp]
        L.shg_batch_plan_launch.restype = ctypes.c_int
        L.shg_batch_plan_powers.argtypes = [vp, ctypes.POINTER(ctypes.c_double), vp]
        L.shg_batch_plan_powers.restype = ctypes.c_int
        L.shg_batch_plan_destroy.argtypes = [vp]
        L.shg_batch_plan_destroy.restype = None
        L.shg_thermal_grad.argtypes = [P, ctypes.POINTER(ShgThermalGradResult)]
        L.shg_thermal_grad.restype = ctypes.c_int
        L.shg_autotune.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(ShgTuneResult)]
        L.shg_autotune.restype = ctypes.c_int
        L.shg_autotune_batch.argtypes = [P, ctypes.c_int32, ctypes.POINTER(ShgTuneResult), ctypes.c_int32,
                                         ctypes.POINTER(ctypes.c_int32)]
        L.shg_autotune_batch.restype = ctypes.c_int
        L.shg_autotune_reset.argtypes = []
        L.shg_autotune_reset.restype = None
        L.shg_set_schedule.argtypes = [ctypes.c_int32] * 4
        L.shg_set_schedule.restype = ctypes.c_int
        L.shg_reserve_device_memory.argtypes = [ctypes.c_int64]
        L.shg_reserve_device_memory.restype = ctypes.c_int
        L.shg_last_error.restype = ctypes.c_char_p
        L.shg_status_string.argtypes = [ctypes.c_int32]
        L.shg_status_string.restype = ctypes.c_char_p
        L.shg_version.restype = ctypes.c_char_p
        _lib = L
    return _lib


def _check(rc: int) -> None:
    if rc != SHG_OK:
        raise ShgError(rc, lib().shg_last_error().decode())


def default_params() -> ShgParams:
    p = ShgParams()
    lib().shg_default_params(ctypes.byref(p))
    return p


def check_params(p: ShgParams) -> int:
    return int(lib().shg_check_params(ctypes.byref(p)))


def fp32_error_estimate(p: ShgParams) -> float:
    """Predicted relative error of the FP32 SH output field (shg_fp32_error_estimate); an
    FP32 instance with ``fp32_guard`` below it runs the FP64 march."""
    return float(lib().shg_fp32_error_estimate(ctypes.byref(p)))


def selftest_bounded_wait(precision: int, wait_us: float, withhold_plane: int) -> None:
    """shg_selftest_bounded_wait: raises ShgError(SHG_ERR_CUDA) when a staged plane's wait ran
    out."""
    _check(lib().shg_selftest_bounded_wait(int(precision), float(wait_us), int(withhold_plane)))


def steps(p: ShgParams) -> int:
    return int(lib().shg_steps(ctypes.byref(p)))


def last_error() -> str:
    return lib().shg_last_error().decode()


def _ptr(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


def solve(p: ShgParams, signal_in: np.ndarray | None = None, want_temperature: bool = False) -> Result:
    """One instance with host buffers (shg_solve)."""
    cdt = p.complex_dtype
    pump = np.empty((p.ny, p.nx), dtype=cdt)
    sig = np.empty((p.ny, p.nx), dtype=cdt)
    T = np.empty((p.nz, p.ny, p.nx), dtype=p.real_dtype) if (want_temperature and p.thermal) else None
    sin = None if signal_in is None else np.ascontiguousarray(np.asarray(signal_in, dtype=cdt).reshape(p.ny, p.nx))
    st = ShgStats()
    _check(lib().shg_solve(ctypes.byref(p), _ptr(sin), _ptr(pump), _ptr(sig), _ptr(T), ctypes.byref(st)))
    return Result(pump=pump, signal=sig, stats=st, temperature=T)


def solve_slices(p: ShgParams, signal_in: np.ndarray | None = None, want_temperature: bool = False):
    """One instance keeping every slice (shg_solve_slices): returns (pump[nz, ny, nx],
    signal[nz, ny, nx], stats, T or None), plane s = the fields before step s."""
    cdt = p.complex_dtype
    pump = np.empty((p.nz, p.ny, p.nx), dtype=cdt)
    sig = np.empty((p.nz, p.ny, p.nx), dtype=cdt)
    T = np.empty((p.nz, p.ny, p.nx), dtype=p.real_dtype) if (want_temperature and p.thermal) else None
    sin = None if signal_in is None else np.ascontiguousarray(np.asarray(signal_in, dtype=cdt).reshape(p.ny, p.nx))
    st = ShgStats()
    _check(lib().shg_solve_slices(ctypes.byref(p), _ptr(sin), _ptr(pump), _ptr(sig), _ptr(T), ctypes.byref(st)))
    return pump, sig, st, T


def run(power: float, waist: float, focalpoint: float, temp: float, t_inf: float, t_peltier: float,
        params: ShgParams | None = None, save_temperature: bool = False) -> Result:
    """``Solver::run`` (src/headers/Solver.h:311) with the crystal / grid of ``params``
    (default: the reference's compile-time configuration)."""
    p = (params or default_params()).copy()
    p.power, p.waist, p.focus = power, waist, focalpoint
    p.temp, p.t_inf, p.t_peltier = temp, t_inf, t_peltier
    return solve(p, want_temperature=save_temperature)


def solve_device(p: ShgParams, pump_out, signal_out, signal_in=None, temperature_out=None, stream=None,
                 stats: bool = True) -> ShgStats | None:
    """One instance on device tensors (torch, complex64/complex128, contiguous)."""
    st = ShgStats() if stats else None

    def dp(t):
        return None if t is None else ctypes.c_void_p(t.data_ptr())

    s = None if stream is None else ctypes.c_void_p(stream)
    _check(lib().shg_solve_device(ctypes.byref(p), dp(signal_in), dp(pump_out), dp(signal_out),
                                  dp(temperature_out), ctypes.byref(st) if st is not None else None, s))
    return st


def solve_batch_device(ps: list[ShgParams], pump_outs=None, signal_outs=None, stream=None,
                       want_power: bool = True) -> np.ndarray | None:
    """Batch of plain instances (shg_solve_batch_device); outputs are device tensors."""
    n = len(ps)
    arr = (ShgParams * n)(*ps)
    vp = ctypes.c_void_p

    def ptrs(ts):
        if ts is None:
            return None
        return (vp * n)(*[vp(t.data_ptr()) if t is not None else None for t in ts])

    power = np.zeros(n, dtype=np.float64) if want_power else None
    pp = power.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if power is not None else None
    s = None if stream is None else vp(stream)
    _check(lib().shg_solve_batch_device(arr, n, ptrs(pump_outs), ptrs(signal_outs), pp, s))
    return power


def heat_sweeps_device(p: ShgParams, temperature, q, sweeps: int, stream=None) -> None:
    """`sweeps` Jacobi sweeps of the heat equation in place on a device tensor
    (shg_heat_sweeps_device); temperature and q are contiguous real tensors of shape
    (nz, ny, nx) in the precision of p."""
    s = None if stream is None else ctypes.c_void_p(stream)
    _check(lib().shg_heat_sweeps_device(ctypes.byref(p), ctypes.c_void_p(temperature.data_ptr()),
                                        ctypes.c_void_p(q.data_ptr()), int(sweeps), s))


def heat_steady_device(p: ShgParams, temperature, q=None, stream=None) -> float:
    """The temperature the Jacobi sweeps converge to, in place on a device tensor
    (shg_heat_steady_device): temperature and q are contiguous real tensors of shape
    (nz, ny, nx) in the precision of p (q None: no heat source); the Dirichlet voxels of
    temperature keep their values.  Returns max |J(T) - T| of one FP64 Jacobi sweep J of the
    FP64 solution."""
    s = None if stream is None else ctypes.c_void_p(stream)
    r = ctypes.c_double(0.0)
    qp = ctypes.c_void_p(q.data_ptr()) if q is not None else None
    _check(lib().shg_heat_steady_device(ctypes.byref(p), ctypes.c_void_p(temperature.data_ptr()), qp,
                                        ctypes.byref(r), s))
    return r.value


def heat_operator_modes(m: int, d: float, lo_robin: bool, hi_robin: bool, bi: float):
    """Eigenvalues, forward and inverse transforms (m x m) of one direction's operator of the
    direct heat solve (shg_heat_operator_modes; host only)."""
    lam = np.zeros(m)
    F = np.zeros((m, m))
    G = np.zeros((m, m))
    dp = ctypes.POINTER(ctypes.c_double)
    _check(lib().shg_heat_operator_modes(int(m), float(d), int(bool(lo_robin)), int(bool(hi_robin)), float(bi),
                                         lam.ctypes.data_as(dp), F.ctypes.data_as(dp), G.ctypes.data_as(dp)))
    return lam, F, G


def _host_ptr(a):
    """Address of a host array: a numpy array or a (pinned) CPU torch tensor; None for None."""
    if a is None:
        return None
    return a.data_ptr() if hasattr(a, "data_ptr") else a.ctypes.data


def solve_batch(ps: list[ShgParams], pumps=None, sigs=None):
    """Batch of plain instances with host buffers (shg_solve_batch).  pumps / sigs: host arrays
    to fill (numpy arrays or pinned torch tensors, one per instance, or None entries for
    outputs not wanted) or None to allocate numpy arrays.  Pinned tensors are written by the
    march directly.  Returns (pumps, sigs, SH powers)."""
    n = len(ps)
    arr = (ShgParams * n)(*ps)
    vp = ctypes.c_void_p
    if pumps is None:
        pumps = [np.empty((p.ny, p.nx), dtype=p.complex_dtype) for p in ps]
    if sigs is None:
        sigs = [np.empty((p.ny, p.nx), dtype=p.complex_dtype) for p in ps]
    power = np.zeros(n, dtype=np.float64)
    _check(lib().shg_solve_batch(arr, n, (vp * n)(*[vp(_host_ptr(a)) for a in pumps]),
                                 (vp * n)(*[vp(_host_ptr(a)) for a in sigs]),
                                 power.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
    return pumps, sigs, power


def _dptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def grad(p: ShgParams, poling: np.ndarray | None = None, checkpoint_every: int = 0) -> dict:
    """Gradients of the SH output power by the adjoint march (shg_grad): returns a dict with
    sh_power, d_waist, d_focus, d_temp, d_poling (array of shg_steps values), device_ms."""
    n = steps(p)
    pol = None if poling is None else np.ascontiguousarray(np.asarray(poling, dtype=np.float64))
    if pol is not None and pol.shape != (n,):
        raise ValueError(f"poling must have {n} values")
    dpol = np.zeros(n, dtype=np.float64)
    r = ShgGradResult()
    r.d_poling = _dptr(dpol)
    _check(lib().shg_grad(ctypes.byref(p), _dptr(pol), int(checkpoint_every), ctypes.byref(r)))
    return {"sh_power": r.sh_power, "d_waist": r.d_waist, "d_focus": r.d_focus, "d_temp": r.d_temp,
            "d_poling": dpol, "device_ms": r.device_ms, "checkpoint_every": r.checkpoint_every, "steps": r.steps}


def grad_batch(ps: list[ShgParams], polings=None, checkpoint_every: int = 0) -> list[dict]:
    """Gradients of many plain runs in one launch (shg_grad_batch); polings: None or a list of
    per-instance poling vectors (entries may be None).  checkpoint_every <= 0: every step's
    fields are kept when the batch covers every SM and they fit in half the free device
    memory, else about sqrt(steps).  Returns one dict per instance as grad."""
    n = len(ps)
    arr = (ShgParams * n)(*ps)
    DP = ctypes.POINTER(ctypes.c_double)
    keep = []
    pol_arr = None
    if polings is not None:
        pol_arr = (DP * n)()
        for i, v in enumerate(polings):
            if v is not None:
                a = np.ascontiguousarray(np.asarray(v, dtype=np.float64))
                if a.shape != (steps(ps[i]),):
                    raise ValueError(f"poling {i} must have {steps(ps[i])} values")
                keep.append(a)
                pol_arr[i] = _dptr(a)
    res = (ShgGradResult * n)()
    dpols = []
    for i in range(n):
        d = np.zeros(steps(ps[i]), dtype=np.float64)
        dpols.append(d)
        res[i].d_poling = _dptr(d)
    _check(lib().shg_grad_batch(arr, n, pol_arr, int(checkpoint_every), res))
    return [{"sh_power": r.sh_power, "d_waist": r.d_waist, "d_focus": r.d_focus, "d_temp": r.d_temp,
             "d_poling": dpols[i], "device_ms": r.device_ms, "checkpoint_every": r.checkpoint_every,
             "steps": r.steps} for i, r in enumerate(res)]


def sh_power(p: ShgParams, poling: np.ndarray | None = None) -> float:
    """SH output power of a plain run with an optional per-step poling phase (shg_sh_power)."""
    pol = None if poling is None else np.ascontiguousarray(np.asarray(poling, dtype=np.float64))
    out = ctypes.c_double(0.0)
    _check(lib().shg_sh_power(ctypes.byref(p), _dptr(pol), ctypes.byref(out)))
    return float(out.value)


NOALLOC_MAX_INSTANCES = 64


def solve_batch_device_noalloc(ps: list[ShgParams], pump_outs=None, signal_outs=None, stream=None,
                               want_power: bool = True) -> np.ndarray | None:
    """shg_solve_batch_device_noalloc: the batched march with no device allocation, for
    callers that cannot allocate while they run.  Its scratch is a fixed array inside the
    library shared by all calls: at most 64 instances per call, and calls that overlap on the
    GPU race.  Outputs are device tensors."""
    n = len(ps)
    arr = (ShgParams * n)(*ps)
    vp = ctypes.c_void_p

    def ptrs(ts):
        if ts is None:
            return None
        return (vp * n)(*[vp(t.data_ptr()) if t is not None else None for t in ts])

    power = np.zeros(n, dtype=np.float64) if want_power else None
    pp = power.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if power is not None else None
    s = None if stream is None else vp(stream)
    _check(lib().shg_solve_batch_device_noalloc(arr, n, ptrs(pump_outs), ptrs(signal_outs), pp, s))
    return power


class BatchPlan:
    """A batched march captured into a CUDA graph (shg_batch_plan_*): create once for a list
    of parameter sets and device output tensors, then ``launch`` replays it on a stream and
    ``powers`` reads the SH powers of the last finished replay."""

    def __init__(self, ps: list[ShgParams], pump_outs=None, signal_outs=None):
        n = len(ps)
        self.count = n
        arr = (ShgParams * n)(*ps)
        vp = ctypes.c_void_p

        def ptrs(ts):
            if ts is None:
                return None
            return (vp * n)(*[vp(t.data_ptr()) if t is not None else None for t in ts])

        self._keep = (pump_outs, signal_outs)
        self._h = vp()
        _check(lib().shg_batch_plan_create(arr, n, ptrs(pump_outs), ptrs(signal_outs), ctypes.byref(self._h)))

    def launch(self, stream=None) -> None:
        _check(lib().shg_batch_plan_launch(self._h, None if stream is None else ctypes.c_void_p(stream)))

    def powers(self, stream=None) -> np.ndarray:
        out = np.zeros(self.count, dtype=np.float64)
        _check(lib().shg_batch_plan_powers(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                           None if stream is None else ctypes.c_void_p(stream)))
        return out

    def close(self) -> None:
        if self._h:
            lib().shg_batch_plan_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def thermal_batch(ps: list[ShgParams], pump_outs=None, signal_outs=None, temperature_outs=None, grad: bool = False,
                  stream=None) -> tuple[list[ShgStats], np.ndarray | None]:
    """shg_thermal_batch: thermal runs in lockstep with batched optical (and, with grad, tangent)
    passes; outputs are device tensors (or None).  Returns the per-instance stats and, with grad,
    dJ/dT_oven per instance."""
    n = len(ps)
    arr = (ShgParams * n)(*ps)
    vp = ctypes.c_void_p

    def ptrs(ts):
        if ts is None:
            return None
        return (vp * n)(*[vp(t.data_ptr()) if t is not None else None for t in ts])

    stats = (ShgStats * n)()
    dt = np.zeros(n, dtype=np.float64) if grad else None
    dp = dt.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if dt is not None else None
    s = None if stream is None else vp(stream)
    _check(lib().shg_thermal_batch(arr, n, ptrs(pump_outs), ptrs(signal_outs), ptrs(temperature_outs), stats, dp, s))
    return list(stats), dt


def thermal_grad(p: ShgParams) -> dict:
    """shg_thermal_grad: a thermal run and dJ/dT_oven through its temperature field."""
    r = ShgThermalGradResult()
    _check(lib().shg_thermal_grad(ctypes.byref(p), ctypes.byref(r)))
    return {"sh_power": r.sh_power, "d_temp": r.d_temp, "sh_power_tangent_march": r.sh_power_tangent_march,
            "device_ms": r.device_ms, "jacobi_sweeps": r.stats.jacobi_sweeps,
            "outer_iterations": r.stats.outer_iterations, "jacobi_ms": r.stats.jacobi_ms,
            "optics_ms": r.stats.optics_ms}


def autotune(precision: int, n: int) -> dict:
    """shg_autotune: time every compiled variant of the (precision, n) class and use the
    fastest from now on; returns the choice and the rates."""
    r = ShgTuneResult()
    _check(lib().shg_autotune(int(precision), int(n), ctypes.byref(r)))
    return {"precision": r.precision, "n": r.n, "cluster": r.cluster, "threads": r.threads,
            "candidates": r.candidates, "pt_steps_per_s": r.pt_steps_per_s,
            "default_pt_steps_per_s": r.default_pt_steps_per_s}


def autotune_reset() -> None:
    """shg_autotune_reset: back to the compiled default schedules."""
    lib().shg_autotune_reset()


def reserve_device_memory(nbytes: int) -> None:
    """shg_reserve_device_memory: grow the library's pool to hold nbytes and keep them."""
    _check(lib().shg_reserve_device_memory(int(nbytes)))


def set_schedule(precision: int, n: int, cluster: int, threads: int) -> None:
    """shg_set_schedule: use the compiled variant of (precision, n) with this split."""
    _check(lib().shg_set_schedule(int(precision), int(n), int(cluster), int(threads)))


def autotune_batch(ps: list[ShgParams]) -> list[dict]:
    """shg_autotune_batch: the launch schedule of every grid-size class of this batch, chosen
    by the time of the whole batch; one dict per class (largest work first) as autotune()."""
    n = len(ps)
    arr = (ShgParams * n)(*ps)
    out = (ShgTuneResult * 16)()
    k = ctypes.c_int32(0)
    _check(lib().shg_autotune_batch(arr, n, out, 16, ctypes.byref(k)))
    return [{"precision": r.precision, "n": r.n, "cluster": r.cluster, "threads": r.threads,
             "candidates": r.candidates, "pt_steps_per_s": r.pt_steps_per_s,
             "default_pt_steps_per_s": r.default_pt_steps_per_s} for r in out[:k.value]]
