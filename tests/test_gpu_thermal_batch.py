"""Batched thermal runs (shg_thermal_batch) through the C ABI.

The batch replaces the reference's one-process-per-point sweep of thermal runs
(src/cuSHG.sh:58-94 over Solver::run with -DTHERMAL, src/headers/Solver.h:321-373): every outer
iteration runs each instance's Jacobi loop, then one optical pass over the instances still
iterating.  Each instance must equal its own shg_solve run bit for bit (fields, temperature, SH
power, sweep and outer-iteration counts), also when the instances stop after different numbers
of outer iterations; with gradients, each dJ/dT_oven must equal shg_thermal_grad's bit for bit.
"""
import numpy as np
import pytest

from cushg_b200 import params as P
from cushg_b200 import shg

pytestmark = pytest.mark.gpu


def instances(n, nz, precision, temps, rule=P.SHG_CONV_MAXABS):
    out = []
    for t in temps:
        p = P.workload(n, nz, 6000.0, 25.0, 30.0, 3000.0, t, precision=precision, thermal=1)
        p.alpha_p, p.alpha_s, p.beta_s = 2e-5, 1e-4, 1e-3
        p.max_outer = 4
        p.conv_rule = rule
        if rule == P.SHG_CONV_FIXED:
            p.max_sweeps = 40
            p.max_outer = 2
        else:
            p.check_every = 50
            p.jacobi_tol = 2e-4
        out.append(p)
    return out


def run_batch(ps, grad=False):
    import torch
    cdt = torch.complex64 if ps[0].precision == 32 else torch.complex128
    rdt = torch.float32 if ps[0].precision == 32 else torch.float64
    pumps = [torch.empty((p.ny, p.nx), dtype=cdt, device="cuda") for p in ps]
    sigs = [torch.empty((p.ny, p.nx), dtype=cdt, device="cuda") for p in ps]
    temps = [torch.empty((p.nz, p.ny, p.nx), dtype=rdt, device="cuda") for p in ps]
    stats, dt = shg.thermal_batch(ps, pumps, sigs, temps, grad=grad)
    torch.cuda.synchronize()
    return ([t.cpu().numpy() for t in pumps], [t.cpu().numpy() for t in sigs], [t.cpu().numpy() for t in temps], stats,
            dt)


@pytest.mark.parametrize("n,precision", [(64, 64), (128, 32), (256, 64)])
def test_thermal_batch_equals_single_runs(n, precision):
    ps = instances(n, 10, precision, [31.0, 38.0, 45.0])
    pumps, sigs, temps, stats, _ = run_batch(ps)
    outers = set()
    for i, p in enumerate(ps):
        r = shg.solve(p, want_temperature=True)
        assert np.array_equal(pumps[i], r.pump), i
        assert np.array_equal(sigs[i], r.signal), i
        assert np.array_equal(temps[i], r.temperature), i
        assert stats[i].sh_power == r.stats.sh_power, i
        assert stats[i].jacobi_sweeps == r.stats.jacobi_sweeps, i
        assert stats[i].outer_iterations == r.stats.outer_iterations, i
        outers.add(r.stats.outer_iterations)


def test_thermal_batch_multipass_512_fp32():
    ps = instances(512, 6, 32, [30.0, 47.5], rule=P.SHG_CONV_FIXED)
    pumps, sigs, temps, stats, _ = run_batch(ps)
    for i, p in enumerate(ps):
        r = shg.solve(p, want_temperature=True)
        assert np.array_equal(sigs[i], r.signal), i
        assert np.array_equal(temps[i], r.temperature), i
        assert stats[i].sh_power == r.stats.sh_power, i


@pytest.mark.parametrize("n", [256, 512])
def test_thermal_batch_gradients_equal_single_gradients(n):
    ps = instances(n, 8, 64 if n == 256 else 32, [33.0, 41.0], rule=P.SHG_CONV_FIXED)
    _, _, _, stats, dt = run_batch(ps, grad=True)
    for i, p in enumerate(ps):
        g = shg.thermal_grad(p)
        assert stats[i].sh_power == g["sh_power"], i
        assert dt[i] == g["d_temp"], i


def test_thermal_batch_rejects_mixed_grids():
    ps = instances(64, 10, 64, [31.0]) + instances(128, 10, 64, [31.0])
    with pytest.raises(shg.ShgError) as e:
        shg.thermal_batch(ps)
    assert e.value.status == P.SHG_ERR_INVALID
