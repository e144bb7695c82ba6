"""Adjoint gradients of the SH output power (shg_grad) against central finite differences of
the forward march, in FP64, and FP32 against FP64.

The forward model with a per-step poling phase is first checked against the oracle; the
gradients must match central differences to 1e-5 relative (FP64), and the FP32 adjoint
the FP64 adjoint and FP64 central differences to 1e-4 (relative to each gradient's scale)."""
import numpy as np
import pytest

from cushg_b200 import params as P
from cushg_b200 import shg
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def case(n=64, nz=31, precision=64):
    p = P.workload(n, nz, 10000.0, 20.0, 28.0, 4000.0, 27.5, precision=precision)
    p.lx = p.ly = 12 * 28.0
    return p


def poling_vector(p, seed=3, sigma=0.1):
    return np.random.default_rng(seed).normal(0.0, sigma, size=p.nz - 1)


def test_forward_with_poling_matches_oracle():
    p = case()
    pol = poling_vector(p)
    j = shg.sh_power(p, pol)
    rc, pump, sig, st, _ = O.solve(p, poling=pol)
    assert rc == 0
    assert abs(j - st.sh_power) / st.sh_power <= 1e-12
    # and the poling phase matters
    assert abs(j - shg.sh_power(p)) / j > 1e-4


def fd(f, x, h):
    return (f(x + h) - f(x - h)) / (2 * h)


@pytest.mark.parametrize("n", [64, 128])
def test_fp64_adjoint_matches_finite_differences(n):
    p = case(n)
    pol = poling_vector(p)
    g = shg.grad(p, pol, checkpoint_every=5)
    assert abs(g["sh_power"] - shg.sh_power(p, pol)) / g["sh_power"] <= 1e-12
    dw = fd(lambda w: shg.sh_power(p.replace(waist=w), pol), p.waist, 1e-5 * p.waist)
    df = fd(lambda f: shg.sh_power(p.replace(focus=f), pol), p.focus, 1e-5 * p.lz)
    dT = fd(lambda t: shg.sh_power(p.replace(temp=t, t_peltier=t), pol), p.temp, 1e-4)
    assert abs(g["d_waist"] - dw) <= 1e-5 * abs(dw)
    assert abs(g["d_focus"] - df) <= 1e-5 * abs(df) + 1e-9 * abs(dw)
    assert abs(g["d_temp"] - dT) <= 1e-5 * abs(dT)
    scale = np.abs(g["d_poling"]).max()
    for s in (0, 7, p.nz // 2, p.nz - 2):
        def f(v, s=s):
            q = pol.copy()
            q[s] = v
            return shg.sh_power(p, q)
        assert abs(g["d_poling"][s] - fd(f, pol[s], 1e-6)) <= 1e-5 * scale


def test_checkpoint_interval_does_not_change_gradients():
    p = case()
    pol = poling_vector(p)
    ref = shg.grad(p, pol, checkpoint_every=1)
    for k in (4, 7, p.nz - 1):
        g = shg.grad(p, pol, checkpoint_every=k)
        for key in ("sh_power", "d_waist", "d_focus", "d_temp"):
            assert abs(g[key] - ref[key]) <= 1e-12 * abs(ref[key]) + 1e-300, key
        assert np.allclose(g["d_poling"], ref["d_poling"], rtol=0, atol=1e-12 * np.abs(ref["d_poling"]).max())


@pytest.mark.parametrize("n", [128, 256])
def test_fp32_adjoint_close_to_fp64_and_fd(n):
    p = case(n)
    pol = poling_vector(p)
    g64 = shg.grad(p, pol)
    g32 = shg.grad(p.replace(precision=32), pol)
    for key in ("sh_power", "d_waist", "d_focus", "d_temp"):
        assert abs(g32[key] - g64[key]) <= 1e-4 * abs(g64[key]), key
    scale = np.abs(g64["d_poling"]).max()
    assert np.abs(g32["d_poling"] - g64["d_poling"]).max() <= 1e-4 * scale
    dw = fd(lambda w: shg.sh_power(p.replace(waist=w), pol), p.waist, 1e-6 * p.waist)
    dT = fd(lambda t: shg.sh_power(p.replace(temp=t, t_peltier=t), pol), p.temp, 1e-6 * p.temp)
    assert abs(g32["d_waist"] - dw) <= 1e-4 * abs(dw)
    assert abs(g32["d_temp"] - dT) <= 1e-4 * abs(dT)


def test_torch_autograd_binding_gradcheck():
    import torch
    from cushg_b200.autograd import SHGPower

    p = case(64, nz=11)
    w = torch.tensor(p.waist, dtype=torch.float64, requires_grad=True)
    f = torch.tensor(p.focus, dtype=torch.float64, requires_grad=True)
    t = torch.tensor(p.temp, dtype=torch.float64, requires_grad=True)
    pol = torch.tensor(poling_vector(p), dtype=torch.float64, requires_grad=True)
    j = SHGPower.apply(w, f, t, pol, p)
    j.backward()
    g = shg.grad(p, pol.detach().numpy())
    assert w.grad.item() == g["d_waist"] and t.grad.item() == g["d_temp"]
    # torch's own finite-difference check of the binding (poling entries and temperature)
    fn = lambda tt, pp: SHGPower.apply(w.detach(), f.detach(), tt, pp, p)  # noqa: E731
    assert torch.autograd.gradcheck(fn, (t, pol), eps=1e-6, atol=1e-12, rtol=1e-4)


def test_grad_batch_equals_single_gradients():
    """Several instances (different nz, power, focus and poling) in one batched launch give
    each instance's shg_grad result."""
    ps, pols = [], []
    for i, nz in enumerate((31, 17, 24)):
        p = case(64, nz=nz).replace(power=10.0 + 5 * i, focus=2000.0 + 1500.0 * i)
        ps.append(p)
        pols.append(poling_vector(p, seed=i) if i != 1 else None)
    got = shg.grad_batch(ps, pols, checkpoint_every=6)
    for p, pol, g in zip(ps, pols, got):
        ref = shg.grad(p, pol, checkpoint_every=6)
        for key in ("sh_power", "d_waist", "d_focus", "d_temp"):
            assert g[key] == ref[key], key
        assert np.array_equal(g["d_poling"], ref["d_poling"])


def test_batch_filling_the_gpu_keeps_every_step():
    """With checkpoint_every <= 0, a batch whose clusters cover every SM keeps every step's
    fields (no re-march), a small batch about sqrt(steps); both give the gradients of an
    explicit interval to round-off."""
    ps, pols = [], []
    for i in range(160):
        p = case(64, nz=13).replace(power=10.0 + 0.1 * i)
        ps.append(p)
        pols.append(poling_vector(p, seed=i))
    auto = shg.grad_batch(ps, pols)
    fixed = shg.grad_batch(ps, pols, checkpoint_every=3)
    for a, f in zip(auto, fixed):
        assert a["checkpoint_every"] == a["steps"] == 12 and f["checkpoint_every"] == 3
        for key in ("sh_power", "d_waist", "d_focus", "d_temp"):
            assert abs(a[key] - f[key]) <= 1e-12 * abs(f[key]) + 1e-300, key
        assert np.allclose(a["d_poling"], f["d_poling"], rtol=0, atol=1e-12 * np.abs(f["d_poling"]).max())
    small = shg.grad_batch(ps[:2], pols[:2])
    assert all(r["checkpoint_every"] == 3 for r in small)  # round(sqrt(12))
