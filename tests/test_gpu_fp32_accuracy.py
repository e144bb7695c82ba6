"""Accuracy of the FP32 batched sweep against the FP64 march, through the C ABI.

The workload is the 256-instance parameter sweep (grid sides 64-256, nz 100-400, P 1-50 W,
w0 15-60 µm, focus anywhere, oven 20-80 °C, L 10 or 20 mm).  With fp32_guard = g every
instance whose predicted FP32 SH field error (shg_fp32_error_estimate) exceeds g runs the FP64
march with FP32 outputs.  The bench's setting g = 1e-5 keeps every instance of seed 0 within
1e-5 relative SH power of the FP64 march (measured 7.1e-6).  Over seeds 1-5 it leaves 3 of
1280 instances between 1e-5 and 1.2e-5: the estimate follows the measured field error with a
spread of about 1.6x (90th percentile), and the power's relative error reaches about 1.5x the
field's.  g = 5e-6 keeps all of them within 1e-5.  A promoted instance's outputs are the
FP64 march's fields rounded to FP32, bit for bit, and a single solve equals its batch
instance bit for bit.
"""
import numpy as np
import pytest

from cushg_b200 import params as P
from cushg_b200 import shg

pytestmark = pytest.mark.gpu

GUARD = 1e-5        # the bench's setting
TIGHT_GUARD = 5e-6  # every seed of 0-5 within 1e-5


def sweep(precision, guard=0.0, seed=0):
    return [p.replace(precision=precision, fp32_guard=guard) for p in P.config_sweep(256, seed=seed)]


def test_guarded_fp32_sweep_meets_1e5_sh_power_on_every_instance():
    import torch
    p32 = sweep(32, GUARD)
    p64 = sweep(64)
    promoted = [i for i, p in enumerate(p32) if shg.fp32_error_estimate(p) > GUARD]
    # the guard promotes about a tenth of the sweep's work
    work = np.array([p.nx * p.nx * (p.nz - 1) for p in p32], dtype=np.float64)
    assert 0 < len(promoted) < 40 and work[promoted].sum() < 0.15 * work.sum()
    s32 = [torch.empty((p.ny, p.nx), dtype=torch.complex64, device="cuda") for p in p32]
    s64 = [torch.empty((p.ny, p.nx), dtype=torch.complex128, device="cuda") for p in p64]
    w32 = shg.solve_batch_device(p32, None, s32)
    w64 = shg.solve_batch_device(p64, None, s64)
    torch.cuda.synchronize()
    rel = np.abs(w32 - w64) / np.abs(w64)
    assert rel.max() <= 1e-5, (int(rel.argmax()), float(rel.max()))
    for i in promoted:
        assert torch.equal(s32[i], s64[i].to(torch.complex64)), i
    # the same instances without the guard: all FP32
    w_plain = shg.solve_batch_device(sweep(32), None, None)
    assert not np.array_equal(w_plain[promoted], w32[promoted])
    keep = [i for i in range(len(p32)) if i not in promoted]
    assert np.array_equal(w_plain[keep], w32[keep])


@pytest.mark.parametrize("seed", [1, 2, 3, 4, 5])
def test_guarded_fp32_sweeps_of_other_seeds_meet_1e5(seed):
    w32 = shg.solve_batch_device(sweep(32, TIGHT_GUARD, seed), None, None)
    w64 = shg.solve_batch_device(sweep(64, 0.0, seed), None, None)
    rel = np.abs(w32 - w64) / np.abs(w64)
    assert rel.max() <= 1e-5, (int(rel.argmax()), float(rel.max()))


def test_guarded_single_solve_equals_its_batch_instance():
    p32 = sweep(32, GUARD)
    i = max(range(len(p32)), key=lambda k: shg.fp32_error_estimate(p32[k]) if p32[k].nx <= 128 else 0.0)
    p = p32[i]
    assert shg.fp32_error_estimate(p) > GUARD
    r = shg.solve(p)
    assert r.signal.dtype == np.complex64
    import torch
    b = [torch.empty((q.ny, q.nx), dtype=torch.complex64, device="cuda") for q in (p, p32[0])]
    pw = shg.solve_batch_device([p, p32[0]], None, b)
    torch.cuda.synchronize()
    assert np.array_equal(b[0].cpu().numpy(), r.signal)
    assert pw[0] == r.sh_power
    r64 = shg.solve(p.replace(precision=64, fp32_guard=0.0))
    assert np.array_equal(r.signal, r64.signal.astype(np.complex64))
