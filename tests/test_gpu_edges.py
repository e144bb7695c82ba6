"""Edge cases of the march through the C ABI against the oracle: a single SSFM step (nz = 2),
zero pump power, a focus outside the crystal, a beam wider than a quarter of the window,
empty and single-instance batches, signal_in through the multi-pass march, and the largest
built grid side with a long march."""
import numpy as np
import pytest

from cushg_b200 import params as P
from cushg_b200 import shg
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a, np.complex128) - b) / np.linalg.norm(b))


def base(n=64, nz=9, precision=64):
    return P.workload(n, nz, 5000.0, 12.0, 28.0, 2500.0, 31.0, precision=precision)


@pytest.mark.parametrize("n,march", [(64, P.SHG_MARCH_AUTO), (256, P.SHG_MARCH_FUSED), (256, P.SHG_MARCH_MULTIPASS),
                                     (512, P.SHG_MARCH_AUTO)])
def test_single_step(n, march):
    """nz = 2: one SSFM step (the reference's output is taken before its second)."""
    p = base(n, nz=2).replace(march=march)
    r = shg.solve(p)
    rc, pump, sig, st, _ = O.solve(p)
    assert rc == 0 and r.stats.steps == 1
    assert rel_l2(r.pump, pump) <= 1e-10 and rel_l2(r.signal, sig) <= 1e-10


def test_zero_power_gives_zero_fields():
    p = base().replace(power=0.0)
    r = shg.solve(p)
    assert not np.any(r.pump) and not np.any(r.signal) and r.sh_power == 0.0


@pytest.mark.parametrize("focus", [-3000.0, 9000.0])
def test_focus_outside_the_crystal(focus):
    p = base().replace(focus=focus)
    r = shg.solve(p)
    rc, pump, sig, st, _ = O.solve(p)
    assert rc == 0
    assert rel_l2(r.signal, sig) <= 1e-10
    assert abs(r.sh_power - st.sh_power) <= 1e-12 * st.sh_power


def test_wide_beam_reaches_the_window_edges():
    """A waist of a quarter of the window: the field at the edges is not negligible, so the
    transform's periodic wrap is exercised."""
    p = base(128).replace(waist=40.0)
    p.lx = p.ly = 160.0
    r = shg.solve(p)
    rc, pump, sig, st, _ = O.solve(p)
    assert rc == 0
    assert np.abs(r.pump[0]).max() > 1e-3 * np.abs(r.pump).max()
    assert rel_l2(r.pump, pump) <= 1e-10 and rel_l2(r.signal, sig) <= 1e-10


def test_empty_and_single_instance_batches():
    import torch
    assert shg.solve_batch_device([], [], []).shape == (0,)
    p = base()
    out = [torch.empty((p.ny, p.nx), dtype=torch.complex128, device="cuda")]
    sig = [torch.empty_like(out[0])]
    pw = shg.solve_batch_device([p], out, sig)
    r = shg.solve(p)
    assert np.array_equal(sig[0].cpu().numpy(), r.signal) and pw[0] == r.sh_power


def test_signal_in_through_the_multipass_march():
    p = base(512, nz=5)
    rng = np.random.default_rng(4)
    s0 = (rng.normal(size=(p.ny, p.nx)) + 1j * rng.normal(size=(p.ny, p.nx))) * 1e-3
    r = shg.solve(p, signal_in=s0)
    rc, pump, sig, st, _ = O.solve(p, signal_in=s0)
    assert rc == 0
    assert rel_l2(r.signal, sig) <= 1e-10


def test_long_march_at_the_largest_side():
    """512 x 512 with 400 steps (FP32 against FP64): the multi-pass march's error stays at
    the FP32 level over a long march."""
    p = base(512, nz=401, precision=32)
    r32 = shg.solve(p)
    r64 = shg.solve(p.replace(precision=64))
    assert rel_l2(r32.signal, r64.signal) <= 1e-4
    assert abs(r32.sh_power - r64.sh_power) <= 1e-4 * r64.sh_power


def test_reserved_pool_serves_later_runs():
    """shg_reserve_device_memory grows the library's pool; runs after it give the same bits."""
    p = P.workload(128, 12, 6000.0, 10.0, 30.0, 3000.0, 30.0, precision=32)
    before = shg.solve(p)
    shg.reserve_device_memory(1 << 30)
    after = shg.solve(p)
    assert np.array_equal(before.signal, after.signal) and before.sh_power == after.sh_power
