"""The direct heat solve on the GPU (shg_heat_steady_device, heat_solver = SHG_HEAT_DIRECT).

* Against the fixed point of the oracle's Jacobi sweep (dense, small grids): max |ΔT| <= 1e-9 K
  in FP64; in FP32 the stored temperature is that fixed point rounded (<= 1e-5 K at 40 °C).
* On the 128 x 128 x 200 FP64 thermal grid and at 512 x 512 x 64 FP32: the solution is
  a fixed point of the library's own Jacobi sweep (the kernel pinned bit for bit to the
  reference), max |J(T) - T| <= 1e-10 K, and the FP64 residual the solve reports agrees.
* A thermal run with the direct solver equals the Jacobi thermal run converged to 1e-12 K
  (fields relative L2 <= 1e-8, T <= 1e-7 K), and its dJ/dT_oven equals central finite
  differences of direct runs to 1e-5 relative (measured 1.0e-7 at sides 256 and 512).
* The FP32 thermal path (FP32 fields, FP64 heat solve), which the large 512 x 512 x 1000 batch
  runs, against FP64 runs with the same solver: at one full-size instance of that batch,
  T <= 2e-5 K, SH field relative L2 <= 5e-5 and SH power <= 2e-5."""
import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN
from cushg_b200 import params as P
from cushg_b200 import shg
from oracle import golden_cases as G

import heat_ref as H

pytestmark = pytest.mark.gpu


def dev(a, dtype):
    return torch.from_numpy(np.ascontiguousarray(a)).to(dtype).cuda()


@pytest.mark.parametrize("boundary", [P.SHG_BOUNDARY_TOP_OPEN, P.SHG_BOUNDARY_OVEN_SURROUNDED])
@pytest.mark.parametrize("n,nz", [(6, 5), (8, 7), (12, 9)])
@pytest.mark.parametrize("precision", [64, 32])
def test_steady_matches_oracle_fixed_point(boundary, n, nz, precision):
    p, T0, Q = H.small_case(n, nz, boundary, precision=precision)
    dt = torch.float64 if precision == 64 else torch.float32
    if precision == 32:
        Q = Q.astype(np.float32).astype(np.float64)
        T0 = T0.astype(np.float32).astype(np.float64)
    ref = H.fixed_point(p.replace(precision=64), T0, Q)
    T = dev(T0, dt)
    r = shg.heat_steady_device(p, T, dev(Q, dt))
    got = T.cpu().double().numpy()
    tol = 1e-9 if precision == 64 else 1e-5
    assert np.abs(got - ref).max() < tol
    assert r < 1e-10
    # the Dirichlet voxels keep their values
    mask = H.dirichlet_mask(p)
    assert np.array_equal(got[mask], T0[mask])


def test_steady_without_heat_source():
    p, T0, _ = H.small_case(8, 7, P.SHG_BOUNDARY_TOP_OPEN)
    ref = H.fixed_point(p, T0, np.zeros_like(T0))
    T = dev(T0, torch.float64)
    shg.heat_steady_device(p, T, None)
    assert np.abs(T.cpu().numpy() - ref).max() < 1e-9


@pytest.mark.parametrize("n,nz,precision,boundary", [
    (128, 200, 64, P.SHG_BOUNDARY_TOP_OPEN),
    (128, 200, 64, P.SHG_BOUNDARY_OVEN_SURROUNDED),
    (96, 37, 64, P.SHG_BOUNDARY_TOP_OPEN),
    (512, 64, 32, P.SHG_BOUNDARY_TOP_OPEN),
])
def test_steady_is_a_fixed_point_at_size(n, nz, precision, boundary):
    p = P.config_thermal_128().replace(nx=n, ny=n, nz=nz, precision=precision, boundary=boundary)
    dt = torch.float64 if precision == 64 else torch.float32
    g = torch.Generator(device="cuda").manual_seed(1)
    Q = torch.rand((nz, n, n), generator=g, device="cuda", dtype=torch.float64) * (60.0 * p.kappa / p.lx**2)
    T0 = torch.from_numpy(H.initial_temperature(p)).cuda()
    T = T0.to(dt).clone()
    r = shg.heat_steady_device(p, T, Q.to(dt))
    assert r < 1e-10
    assert float((T.double() - T0).abs().max()) > 0.1  # the solve moved the field
    if precision == 64:
        swept = T.clone()
        shg.heat_sweeps_device(p, swept, Q, 1)
        assert float((swept - T).abs().max()) < 1e-10


def thermal_case(solver):
    p = P.workload(32, 16, 5000.0, 25.0, 28.0, 2500.0, 31.0, precision=64, thermal=1)
    p.alpha_p, p.alpha_s, p.beta_s = 2e-5, 1e-4, 1e-3
    p.max_outer = 3
    p.conv_rule = P.SHG_CONV_MAXABS
    p.jacobi_tol = 1e-12
    p.check_every = 200
    p.heat_solver = solver
    return p


def test_thermal_run_direct_equals_converged_jacobi():
    rj = shg.solve(thermal_case(P.SHG_HEAT_JACOBI), want_temperature=True)
    rd = shg.solve(thermal_case(P.SHG_HEAT_DIRECT), want_temperature=True)
    assert rd.stats.outer_iterations == rj.stats.outer_iterations == 3
    assert rd.stats.jacobi_sweeps == 0 and rj.stats.jacobi_sweeps > 1000
    assert rd.stats.last_residual < 1e-10
    assert np.abs(rd.temperature - rj.temperature).max() < 1e-7
    for a, b in ((rd.pump, rj.pump), (rd.signal, rj.signal)):
        assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-8
    assert abs(rd.sh_power - rj.sh_power) / rj.sh_power < 1e-8


@pytest.mark.parametrize("n", [256, 512])
def test_thermal_grad_direct_matches_finite_differences(n):
    """dJ/dT_oven of a thermal run with the direct heat solve (absorption on, three outer
    iterations, so the heat source's tangent feeds two later solves) against central
    differences of whole direct runs."""
    p = P.workload(n, 9, 4000.0, 30.0, 25.0, 2000.0, 34.0, precision=64, thermal=1)
    p.alpha_p, p.alpha_s, p.beta_s = 2e-5, 1e-4, 1e-3
    p.conv_rule = P.SHG_CONV_FIXED
    p.max_sweeps = 1  # ignored by the direct solver
    p.max_outer = 3
    p.heat_solver = P.SHG_HEAT_DIRECT
    g = shg.thermal_grad(p)
    assert g["jacobi_sweeps"] == 0 and g["outer_iterations"] == 3
    h = 1e-3

    def run(t):
        return shg.solve(p.replace(temp=t, t_peltier=t)).sh_power

    fd = (run(p.temp + h) - run(p.temp - h)) / (2 * h)
    print(f"n = {n}: dJ/dT_oven {g['d_temp']:.9g}, central differences {fd:.9g}, "
          f"relative {abs(g['d_temp'] - fd) / abs(fd):.3g}")
    assert abs(g["d_temp"] - fd) <= 1e-5 * abs(fd)
    assert abs(g["sh_power"] - run(p.temp)) <= 1e-12 * g["sh_power"]


def fp32_vs_fp64(p):
    r64 = shg.solve(p.replace(precision=64), want_temperature=True)
    r32 = shg.solve(p.replace(precision=32), want_temperature=True)
    dT = float(np.abs(r32.temperature.astype(np.float64) - r64.temperature).max())
    sig = float(np.linalg.norm(r32.signal.astype(np.complex128) - r64.signal) / np.linalg.norm(r64.signal))
    pw = abs(r32.sh_power - r64.sh_power) / r64.sh_power
    print(f"FP32 vs FP64 (direct heat solve): max |dT| {dT:.3g} K, signal rel L2 {sig:.3g}, SH power rel {pw:.3g}")
    assert r32.stats.outer_iterations == r64.stats.outer_iterations
    return dT, sig, pw


def test_thermal_fp32_direct_against_fp64_direct():
    """The FP32 thermal path with the FP64 heat solve against the FP64 run with the same
    solver: the temperature differs by the FP32 optics' effect on Q and the final rounding."""
    dT, sig, pw = fp32_vs_fp64(thermal_case(P.SHG_HEAT_DIRECT))
    # measured: 1.2e-5 K, 3.1e-6, 7.3e-7
    assert dT <= 1e-4
    assert sig <= 3e-5
    assert pw <= 1e-5


def test_large_thermal_instance_fp32_against_fp64():
    """One instance of the large thermal batch as stated (512 x 512, nz = 1000, 50 W,
    w0 = 50 µm, 20 mm, oven 30 °C, max |ΔT| < 1e-6 K, <= 5 outer iterations), FP32 fields
    against FP64 fields, both with the direct heat solve."""
    p = P.config_thermal_512(1)[0].replace(heat_solver=P.SHG_HEAT_DIRECT)
    dT, sig, pw = fp32_vs_fp64(p)
    # measured: 2.2e-6 K, 5.7e-6, 3.8e-6
    assert dT <= 2e-5
    assert sig <= 5e-5
    assert pw <= 2e-5


def test_thermal_128x128x200_direct_against_reference_jacobi():
    """The 128 x 128 x 200 FP64 thermal run (5 outer iterations, Jacobi to max |ΔT| < 1e-6 K)
    with the direct heat solve, against the reference's own run (tests/golden/thermal64_c2.npz).
    They differ by the reference loop's stopping error: its last sweep moves T by less than
    1e-6 K, but the iterate is still that sweep's contraction factor away from the fixed
    point."""
    z = np.load(os.path.join(GOLDEN, "thermal64_c2.npz"))
    p = G.params_of("thermal64_c2").replace(heat_solver=P.SHG_HEAT_DIRECT)
    r = shg.solve(p, want_temperature=True)
    zs = [int(v) for v in z["T_z"]]
    dT = float(np.abs(r.temperature[zs] - z["T_slices"]).max())
    span = float(z["T_max"] - z["T_min"])
    print(f"128 x 128 x 200 thermal run, direct vs the reference's Jacobi: max |dT| {dT:.3g} K on the stored slices "
          f"(T spans {span:.3g} K), {r.stats.outer_iterations} outer iterations, "
          f"FP64 sweep residual {r.stats.last_residual:.3g} K")
    assert r.stats.jacobi_sweeps == 0
    assert r.stats.last_residual < 1e-9
    # measured: 8.45e-3 K of a 0.322 K span
    assert dT < 0.05 * span
