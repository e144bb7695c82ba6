"""The multi-pass SSFM march (field planes in global memory, a row and a column launch per
step) through the C ABI: the same arithmetic as the fused cluster march at 256 x 256, where
both are built (plain and thermal; the two differ only where the compiler contracts a
multiply and an add into one fused multiply-add differently, a last-bit effect), and
matching the CPU oracle at 512 x 512, the side only the multi-pass march runs.

Tolerances: multi-pass against fused, FP64 fields relative L2 <= 1e-13, FP32 <= 1e-5;
against the oracle as in the other parity tests, FP64 fields relative L2 <= 1e-10 and SH
power <= 1e-12, FP32 fields <= 1e-5 against the FP64 oracle."""
import numpy as np
import pytest

from cushg_b200 import params as P
from cushg_b200 import shg
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a, np.complex128) - b) / np.linalg.norm(b))


def case(n, precision, nz=9, seed=0):
    rng = np.random.default_rng(seed)
    waist = float(rng.uniform(20, 45))
    p = P.workload(n, nz, 6000.0, float(rng.uniform(5, 40)), waist, float(rng.uniform(0, 6000.0)),
                   float(rng.uniform(25, 45)), precision=precision)
    p.rho_p, p.rho_s = float(rng.uniform(0, 0.01)), float(rng.uniform(0, 0.01))
    p.ly = p.lx * 0.9
    return p


@pytest.mark.parametrize("precision", [64, 32])
def test_multipass_equals_fused(precision):
    p = case(256, precision, nz=11)
    a = shg.solve(p.replace(march=P.SHG_MARCH_FUSED))
    b = shg.solve(p.replace(march=P.SHG_MARCH_MULTIPASS))
    tol = 1e-13 if precision == 64 else 1e-5
    assert rel_l2(b.signal, a.signal) <= tol and rel_l2(b.pump, a.pump) <= tol
    assert abs(a.sh_power - b.sh_power) <= (1e-12 if precision == 64 else 1e-5) * a.sh_power


@pytest.mark.parametrize("n", [256, 128])
@pytest.mark.parametrize("precision", [64, 32])
def test_multipass_thermal_equals_fused(precision, n):
    p = P.workload(n, 10, 4000.0, 20.0, 25.0, 2000.0, 30.0, precision=precision, thermal=1)
    p.alpha_p, p.alpha_s, p.beta_s = 2e-5, 1e-4, 1e-3
    p.max_outer = 2
    p.check_every = 50
    p.conv_rule = P.SHG_CONV_MAXABS
    p.jacobi_tol = 1e-3
    p.max_sweeps = 20000
    a = shg.solve(p.replace(march=P.SHG_MARCH_FUSED), want_temperature=True)
    b = shg.solve(p.replace(march=P.SHG_MARCH_MULTIPASS), want_temperature=True)
    assert a.stats.outer_iterations == b.stats.outer_iterations
    assert abs(a.stats.jacobi_sweeps - b.stats.jacobi_sweeps) <= p.check_every
    tol_t = 1e-9 if precision == 64 else 1e-3
    assert np.max(np.abs(a.temperature - b.temperature)) <= tol_t
    tol = 1e-10 if precision == 64 else 1e-4
    assert rel_l2(b.signal, a.signal) <= tol and rel_l2(b.pump, a.pump) <= tol
    assert a.sh_power > 0 and abs(b.sh_power - a.sh_power) <= tol * a.sh_power
    assert abs(b.stats.pump_power - a.stats.pump_power) <= tol * a.stats.pump_power


def test_multipass_512_fp64_matches_oracle():
    p = case(512, 64, nz=7, seed=5)
    r = shg.solve(p)
    rc, pump, sig, st, _ = O.solve(p)
    assert rc == 0
    assert rel_l2(r.pump, pump) <= 1e-10
    assert rel_l2(r.signal, sig) <= 1e-10
    assert abs(r.sh_power - st.sh_power) <= 1e-12 * st.sh_power


def test_multipass_512_fp32_against_fp64_oracle():
    p = case(512, 32, nz=7, seed=6)
    r = shg.solve(p)
    rc, pump, sig, st, _ = O.solve(p.replace(precision=64))
    assert rc == 0
    assert rel_l2(r.signal, sig) <= 1e-5
    assert abs(r.sh_power - st.sh_power) <= 1e-5 * st.sh_power


def test_multipass_slices_end_with_outputs():
    p = case(512, 64, nz=4, seed=7)
    pump_sl, sig_sl, st, _ = shg.solve_slices(p)
    r = shg.solve(p)
    assert np.array_equal(pump_sl[-1], r.pump) and np.array_equal(sig_sl[-1], r.signal)
    # plane nz-2: the fields after nz-2 steps of the same dz
    pump0 = np.ascontiguousarray(O.set_pump(p, p.temp).reshape(p.ny, p.nx).astype(np.complex128))
    sig0 = np.zeros_like(pump0)
    O.march_plain(p, p.nz - 2, pump0, sig0)
    assert rel_l2(pump_sl[-2], pump0) <= 1e-10
    assert rel_l2(sig_sl[-2], sig0) <= 1e-10


def test_batch_mixes_fused_and_multipass():
    import torch
    ps = [case(512, 64, nz=5, seed=11), case(256, 64, nz=8, seed=12), case(512, 64, nz=3, seed=13),
          case(128, 64, nz=6, seed=14)]
    pumps = [torch.empty((p.ny, p.nx), dtype=torch.complex128, device="cuda") for p in ps]
    sigs = [torch.empty_like(t) for t in pumps]
    power = shg.solve_batch_device(ps, pumps, sigs)
    for i, p in enumerate(ps):
        r = shg.solve(p)
        assert np.array_equal(sigs[i].cpu().numpy(), r.signal), i
        assert abs(power[i] - r.sh_power) <= 1e-12 * r.sh_power, i
    plan = shg.BatchPlan(ps, pumps, sigs)
    try:
        plan.launch()
        assert np.array_equal(plan.powers(), power)
    finally:
        plan.close()
