"""Parity of the thermal run (Jacobi heat solve + temperature-dependent optics + Q
emission, the reference's -DTHERMAL outer loop) through the C ABI, against the reference's
own FP64 outputs (tests/golden/thermal64_n32*.npz) and the CPU oracle.

Tolerances: fields relative L2 <= 1e-10, temperatures max |ΔT| <= 1e-9 K, SH power 1e-10,
identical Jacobi sweep counts and outer-iteration counts."""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN
from cushg_b200 import params as P
from cushg_b200 import shg
from oracle import golden_cases as G
from oracle import oracle as O

pytestmark = pytest.mark.gpu

THERMAL_GOLDEN = ["thermal64_n32", "thermal64_n32_oven"]


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a, np.complex128) - b) / np.linalg.norm(b))


@pytest.mark.parametrize("name", THERMAL_GOLDEN)
def test_thermal_fp64_matches_reference(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    meta = json.loads(str(z["meta"]))
    p = G.params_of(name)
    r = shg.solve(p, want_temperature=True)
    assert r.stats.jacobi_sweeps == sum(meta["jacobi_sweeps"])
    assert r.stats.outer_iterations == len(meta["jacobi_sweeps"])
    assert np.abs(r.temperature - z["T"]).max() <= 1e-9
    assert rel_l2(r.pump, z["pump"]) <= 1e-10
    assert rel_l2(r.signal, z["signal"]) <= 1e-10


@pytest.mark.parametrize("name", THERMAL_GOLDEN)
def test_thermal_fp64_matches_oracle(name):
    p = G.params_of(name)
    r = shg.solve(p, want_temperature=True)
    rc, pump, sig, st, T = O.solve(p, want_temperature=True)
    assert rc == 0
    assert r.stats.jacobi_sweeps == st.jacobi_sweeps
    assert np.abs(r.temperature - T).max() <= 1e-9
    assert rel_l2(r.signal, sig) <= 1e-10
    # the thermal fields inherit the rounding of tens of thousands of Jacobi sweeps through
    # n(T) and Δk(T), so the power is held to 1e-10 rather than the plain path's 1e-12
    assert abs(r.sh_power - st.sh_power) / st.sh_power <= 1e-10


@pytest.mark.parametrize("n", [64, 128])
def test_thermal_fp64_larger_grids_match_oracle(n):
    p = P.workload(n, 12, 6000.0, 20.0, 30.0, 3000.0, 33.0, precision=64, thermal=1)
    p.alpha_p, p.alpha_s, p.beta_s = 2e-5, 1e-4, 1e-3
    p.max_outer = 2
    p.check_every = 200
    p.conv_rule = P.SHG_CONV_MAXABS
    p.jacobi_tol = 1e-3
    r = shg.solve(p, want_temperature=True)
    rc, pump, sig, st, T = O.solve(p, want_temperature=True)
    assert rc == 0
    assert r.stats.jacobi_sweeps == st.jacobi_sweeps
    assert np.abs(r.temperature - T).max() <= 1e-9
    assert rel_l2(r.signal, sig) <= 1e-10
    assert rel_l2(r.pump, pump) <= 1e-10


def test_thermal_sweep_cap_reports_not_converged():
    p = G.params_of("thermal64_n32").replace(max_sweeps=100)
    with pytest.raises(shg.ShgError) as e:
        shg.solve(p)
    assert e.value.status == P.SHG_ERR_NOT_CONVERGED


def test_thermal_fp32_against_fp64_oracle():
    """FP32 fields and temperatures against the FP64 oracle with the same stopping rule
    (max |ΔT| < 1e-3 K checked every 1000 sweeps, so both stop after the same sweeps)."""
    p = G.params_of("thermal64_n32").replace(conv_rule=P.SHG_CONV_MAXABS, jacobi_tol=1e-3, check_every=1000)
    rc, pump, sig, st, T = O.solve(p, want_temperature=True)
    r = shg.solve(p.replace(precision=32), want_temperature=True)
    assert r.stats.jacobi_sweeps == st.jacobi_sweeps
    # float Jacobi rounding moves T by up to ~1e-2 K after thousands of sweeps, and this
    # off-phase-matched SH is sensitive to Δk(T), so the field bound is percent-level
    assert np.abs(r.temperature - T).max() <= 2e-2
    assert rel_l2(r.signal, sig) <= 2e-2
    assert abs(r.sh_power - st.sh_power) / st.sh_power <= 2e-2


@pytest.mark.parametrize("precision", [64, 32])
@pytest.mark.parametrize("boundary", [P.SHG_BOUNDARY_TOP_OPEN, P.SHG_BOUNDARY_OVEN_SURROUNDED])
@pytest.mark.parametrize("n,nz,check_every", [(64, 50, 8), (32, 23, 7), (128, 40, 30)])
def test_blocked_sweeps_are_bit_identical(precision, boundary, n, nz, check_every):
    """Fusing 2, 3 or 4 sweeps per launch (TMA-staged temporal blocking) gives the same
    temperatures, fields and sweep counts, bit for bit, as one sweep per launch.  The grids
    leave partial tiles at the +x / +y edges and split z into chunks; check windows of
    check_every - 1 unchecked sweeps leave remainders of 1, 2 and 3 sweeps."""
    p = P.workload(n, nz, 6000.0, 3.0, 30.0, 3000.0, 33.0, precision=precision, thermal=1)
    p.alpha_p, p.alpha_s, p.beta_s = 2e-5, 1e-4, 1e-3
    p.boundary = boundary
    p.max_outer = 2
    p.check_every = check_every
    p.conv_rule = P.SHG_CONV_MAXABS
    p.jacobi_tol = 2e-3
    p.max_sweeps = 4000
    ref = shg.solve(p.replace(jacobi_block=1), want_temperature=True)
    for blk in (0, 2, 3, 4):
        r = shg.solve(p.replace(jacobi_block=blk), want_temperature=True)
        assert r.stats.jacobi_sweeps == ref.stats.jacobi_sweeps
        assert r.stats.outer_iterations == ref.stats.outer_iterations
        assert np.array_equal(r.temperature, ref.temperature), blk
        assert np.array_equal(r.signal, ref.signal) and np.array_equal(r.pump, ref.pump)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [64, 32])
@pytest.mark.parametrize("boundary", [P.SHG_BOUNDARY_TOP_OPEN, P.SHG_BOUNDARY_OVEN_SURROUNDED])
@pytest.mark.parametrize("n", [48, 34])
def test_heat_sweeps_match_oracle(precision, boundary, n):
    """shg_heat_sweeps_device (the Tfield::upDate loop) against the oracle's sweep repeated,
    from a random temperature and heat source, for every sweep depth; depths agree bit for
    bit with one sweep per launch.  n = 48: FP32 sweeps take four voxels per thread; n = 34
    (not a multiple of 4): two, and the TMA-staged depths, which need 16-byte rows, refuse
    FP32 (SHG_ERR_UNSUPPORTED)."""
    import torch

    nz, sweeps = 21, 11
    p = P.workload(n, nz, 6000.0, 3.0, 30.0, 3000.0, 33.0, precision=precision, thermal=1)
    p.boundary = boundary
    rng = np.random.default_rng(7)
    rdt = np.float64 if precision == 64 else np.float32
    T0 = (30.0 + 5.0 * rng.random((nz, n, n))).astype(rdt)
    Q = (1e-6 * rng.random((nz, n, n))).astype(rdt)
    Ti, Tf = T0.copy(), T0.copy()
    for _ in range(sweeps):
        O.jacobi_sweep(p, Ti, Q, Tf)
        Ti, Tf = Tf, Ti
    tdt = torch.float64 if precision == 64 else torch.float32
    q_d = torch.from_numpy(Q).to("cuda")
    outs = {}
    rows16 = (n * T0.itemsize) % 16 == 0
    for blk in (1, 2, 3, 4, 0):
        t_d = torch.from_numpy(T0).to("cuda")
        if blk in (2, 3, 4) and not rows16:
            with pytest.raises(shg.ShgError) as e:
                shg.heat_sweeps_device(p.replace(jacobi_block=blk), t_d, q_d, sweeps)
            assert e.value.status == P.SHG_ERR_UNSUPPORTED
            continue
        shg.heat_sweeps_device(p.replace(jacobi_block=blk), t_d, q_d, sweeps)
        torch.cuda.synchronize()
        outs[blk] = t_d.cpu().numpy()
        assert outs[blk].dtype == np.dtype(rdt) and t_d.dtype == tdt
    for blk in outs:
        assert np.array_equal(outs[blk], outs[1]), blk
    tol = 1e-12 if precision == 64 else 2e-6
    assert np.max(np.abs(outs[1] - Ti)) / np.max(np.abs(Ti)) < tol


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [64, 32])
def test_heat_sweeps_reject_misaligned_buffers(precision):
    """The sweep reads voxel pairs: a temperature or Q pointer not aligned to two reals is
    refused on the host (SHG_ERR_INVALID) before anything is launched."""
    import torch

    n, nz = 32, 8
    p = P.workload(n, nz, 6000.0, 3.0, 30.0, 3000.0, 33.0, precision=precision, thermal=1)
    tdt = torch.float64 if precision == 64 else torch.float32
    t_d = torch.full((nz * n * n + 1,), 30.0, dtype=tdt, device="cuda")
    q_d = torch.zeros(nz * n * n + 1, dtype=tdt, device="cuda")
    for t, q in ((t_d[1:], q_d[:-1]), (t_d[:-1], q_d[1:])):
        with pytest.raises(shg.ShgError) as e:
            shg.heat_sweeps_device(p, t, q, 3)
        assert e.value.status == P.SHG_ERR_INVALID
    shg.heat_sweeps_device(p, t_d[:-1], q_d[:-1], 3)  # aligned views run
    torch.cuda.synchronize()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [64, 32])
def test_fixed_sweep_rule_runs_exact_counts(precision):
    """conv_rule FIXED: exactly max_sweeps sweeps per outer iteration and max_outer iterations.
    With one outer iteration the temperature is the initial field (oven on the y = 0 face,
    the phase-matching temperature elsewhere) after max_sweeps sweeps with Q = 0, which is what
    shg_heat_sweeps_device gives from that field."""
    import torch

    p = P.workload(32, 12, 4000.0, 20.0, 25.0, 2000.0, 30.0, precision=precision, thermal=1)
    p.t_peltier = 35.0
    p.conv_rule = P.SHG_CONV_FIXED
    p.max_sweeps = 37
    p.max_outer = 1
    r = shg.solve(p, want_temperature=True)
    assert r.stats.jacobi_sweeps == 37 and r.stats.outer_iterations == 1
    rdt = np.float64 if precision == 64 else np.float32
    T0 = np.full((p.nz, p.ny, p.nx), p.temp, dtype=rdt)
    T0[:, 0, :] = p.t_peltier
    t_d = torch.from_numpy(T0).to("cuda")
    shg.heat_sweeps_device(p, t_d, torch.zeros_like(t_d), 37)
    torch.cuda.synchronize()
    assert np.max(np.abs(t_d.cpu().numpy() - r.temperature)) <= (1e-12 if precision == 64 else 1e-5)
    r2 = shg.solve(p.replace(max_outer=3), want_temperature=True)
    assert r2.stats.jacobi_sweeps == 3 * 37 and r2.stats.outer_iterations == 3


@pytest.mark.parametrize("precision", [32, 64])
def test_blocked_sweep_wait_runs_out_and_reports(precision):
    """The TMA-staged sweeps bound every wait for a staged plane.  With one plane's staging
    withheld and a 20 µs limit the wait runs out: the call returns SHG_ERR_CUDA, the device
    stays usable, and the same sweeps with every plane staged, and a thermal run with blocked
    sweeps, still pass."""
    with pytest.raises(shg.ShgError) as e:
        shg.selftest_bounded_wait(precision, 20.0, 7)
    assert e.value.status == P.SHG_ERR_CUDA
    assert "did not arrive" in str(e.value)
    shg.selftest_bounded_wait(precision, 2e6, -1)
    p = G.params_of("thermal64_n32").replace(jacobi_block=2)
    r = shg.solve(p, want_temperature=True)
    ref = shg.solve(p.replace(jacobi_block=1), want_temperature=True)
    assert np.array_equal(r.temperature, ref.temperature)
