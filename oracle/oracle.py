"""ctypes binding of the CPU oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline / reference legs as the checker.  The product package never imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

from cushg_b200.params import ShgParams, ShgStats

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

_lib = None


def build(force: bool = False) -> str:
    """Compile liboracle.so with the Makefile next to this file."""
    deps = [os.path.join(HERE, f) for f in ("shg_oracle.c", "shg_oracle_impl.h")]
    deps.append(os.path.join(os.path.dirname(HERE), "include", "shg.h"))  # the shared parameter / stats structs
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < max(os.path.getmtime(d) for d in deps):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.POINTER(ShgParams)
        vp = ctypes.c_void_p
        L.shgo_solve.argtypes = [P, vp, vp, vp, vp, ctypes.POINTER(ShgStats)]
        L.shgo_solve.restype = ctypes.c_int
        L.shgo_solve_poling.argtypes = [P, vp, vp, vp, vp, vp, ctypes.POINTER(ShgStats)]
        L.shgo_solve_poling.restype = ctypes.c_int
        L.shgo_march_plain_f64.argtypes = [P, ctypes.c_int, vp, vp]
        L.shgo_march_plain_f32.argtypes = [P, ctypes.c_int, vp, vp]
        L.shgo_batch_plain.argtypes = [P, ctypes.c_int, vp, vp, ctypes.c_int]
        L.shgo_batch_plain.restype = ctypes.c_int
        L.shgo_sellmeier_d.argtypes = [ctypes.c_double, ctypes.c_double]
        L.shgo_sellmeier_d.restype = ctypes.c_double
        L.shgo_crystal_n.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double]
        L.shgo_crystal_n.restype = ctypes.c_double
        L.shgo_delta_k.argtypes = [P, ctypes.c_double]
        L.shgo_delta_k.restype = ctypes.c_double
        L.shgo_set_pump.argtypes = [P, ctypes.c_double, vp]
        L.shgo_propagators.argtypes = [P, ctypes.c_double, vp, vp]
        L.shgo_fft2.argtypes = [ctypes.c_int, vp, ctypes.c_int]
        L.shgo_jacobi_sweep.argtypes = [P, vp, vp, vp]
        L.shgo_jacobi_sweep_f32.argtypes = [P, vp, vp, vp]
        L.shgo_set_q.argtypes = [P, vp, vp, vp, ctypes.c_int, vp]
        L.shgo_sh_power.argtypes = [P, vp, ctypes.c_double]
        L.shgo_sh_power.restype = ctypes.c_double
        L.shgo_set_threads.argtypes = [ctypes.c_int]
        L.shgo_max_threads.restype = ctypes.c_int
        _lib = L
    return _lib


def _ptr(a: np.ndarray | None):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


def set_threads(n: int) -> None:
    lib().shgo_set_threads(int(n))


def max_threads() -> int:
    return int(lib().shgo_max_threads())


def solve(p: ShgParams, signal_in: np.ndarray | None = None, want_temperature: bool = False,
          poling: np.ndarray | None = None):
    """Whole run (plain or thermal).  Returns (pump, signal, stats, T or None).  poling: per-step
    phase [rad] added to the mismatch phase (plain runs)."""
    cdt = p.complex_dtype
    n = p.points
    pump = np.zeros((p.ny, p.nx), dtype=cdt)
    sig = np.zeros((p.ny, p.nx), dtype=cdt)
    T = np.zeros((p.nz, p.ny, p.nx), dtype=p.real_dtype) if (want_temperature and p.thermal) else None
    sin = None
    if signal_in is not None:
        sin = np.ascontiguousarray(signal_in.astype(cdt).reshape(n))
    st = ShgStats()
    pol = None if poling is None else np.ascontiguousarray(np.asarray(poling, dtype=np.float64))
    rc = lib().shgo_solve_poling(ctypes.byref(p), _ptr(sin), _ptr(pol), _ptr(pump), _ptr(sig), _ptr(T),
                                 ctypes.byref(st))
    return rc, pump, sig, st, T


def march_plain(p: ShgParams, steps: int, pump: np.ndarray, signal: np.ndarray) -> None:
    """March `steps` plain SSFM steps in place (complex128 or complex64 arrays)."""
    assert pump.flags.c_contiguous and signal.flags.c_contiguous
    if pump.dtype == np.complex128:
        lib().shgo_march_plain_f64(ctypes.byref(p), int(steps), _ptr(pump), _ptr(signal))
    else:
        lib().shgo_march_plain_f32(ctypes.byref(p), int(steps), _ptr(pump), _ptr(signal))


def batch_plain(ps: list[ShgParams], steps: list[int] | None = None, nthreads: int = 1) -> np.ndarray:
    arr = (ShgParams * len(ps))(*ps)
    st = None if steps is None else np.ascontiguousarray(np.asarray(steps, dtype=np.int32))
    out = np.zeros(len(ps), dtype=np.float64)
    lib().shgo_batch_plain(arr, len(ps), _ptr(st), _ptr(out), int(nthreads))
    return out


def sellmeier(lam: float, temp: float, crystal: int = 0) -> float:
    return float(lib().shgo_crystal_n(crystal, lam, temp))


def delta_k(p: ShgParams, temp: float) -> float:
    return float(lib().shgo_delta_k(ctypes.byref(p), temp))


def set_pump(p: ShgParams, tc: float) -> np.ndarray:
    out = np.zeros((p.ny, p.nx), dtype=np.complex128)
    lib().shgo_set_pump(ctypes.byref(p), tc, _ptr(out))
    return out


def propagators(p: ShgParams, tc: float):
    a = np.zeros((p.ny, p.nx), dtype=np.complex128)
    b = np.zeros((p.ny, p.nx), dtype=np.complex128)
    lib().shgo_propagators(ctypes.byref(p), tc, _ptr(a), _ptr(b))
    return a, b


def fft2(a: np.ndarray, inverse: bool = False) -> np.ndarray:
    out = np.ascontiguousarray(a.astype(np.complex128))
    lib().shgo_fft2(out.shape[0], _ptr(out), 1 if inverse else 0)
    return out


def jacobi_sweep(p: ShgParams, Ti: np.ndarray, Q: np.ndarray, Tf: np.ndarray | None = None) -> np.ndarray:
    if Tf is None:
        Tf = Ti.copy()
    if Ti.dtype == np.float32:
        lib().shgo_jacobi_sweep_f32(ctypes.byref(p), _ptr(Ti), _ptr(Tf), _ptr(Q))
    else:
        lib().shgo_jacobi_sweep(ctypes.byref(p), _ptr(Ti), _ptr(Tf), _ptr(Q))
    return Tf


def set_q(p: ShgParams, T: np.ndarray, P: np.ndarray, S: np.ndarray, s: int, Q: np.ndarray) -> None:
    lib().shgo_set_q(ctypes.byref(p), _ptr(T), _ptr(P), _ptr(S), int(s), _ptr(Q))
