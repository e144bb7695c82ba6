"""The batched march: persistent launches fed by device work queues, batch plans replayed
as CUDA graphs, and the autotuner of the launch schedule, through the C ABI.

Every instance of a batch must come out as the same instance solved alone (the fields are
computed by the same per-point arithmetic whichever cluster takes the instance), and a plan
replay must repeat the direct batch call bit for bit."""
import numpy as np
import pytest

from cushg_b200 import params as P
from cushg_b200 import shg
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def sweep(precision, count, seed, nz_range=(6, 14)):
    rng = np.random.default_rng(seed)
    ps = []
    for i in range(count):
        n = int(rng.choice([32, 64, 128, 192, 256]))
        lz = float(rng.choice([4000.0, 8000.0]))
        waist = float(rng.uniform(15, 40))
        ps.append(P.workload(n, int(rng.integers(*nz_range)), lz, float(rng.uniform(2, 30)), waist,
                             float(rng.uniform(0, lz)), float(rng.uniform(25, 45)), precision=precision))
    return ps


def device_outputs(ps):
    import torch
    dt = torch.complex128 if ps[0].precision == 64 else torch.complex64
    return ([torch.full((p.ny, p.nx), float("nan"), dtype=dt, device="cuda") for p in ps],
            [torch.full((p.ny, p.nx), float("nan"), dtype=dt, device="cuda") for p in ps])


@pytest.mark.parametrize("precision", [64, 32])
def test_batch_instances_equal_single_solves(precision):
    """A batch with more instances than fit on the device at once (so clusters take several
    from the queue), mixed sides and step counts: each instance equals shg_solve of it."""
    import torch
    ps = sweep(precision, 150, seed=precision)
    pumps, sigs = device_outputs(ps)
    power = shg.solve_batch_device(ps, pumps, sigs)
    torch.cuda.synchronize()
    for i in range(0, len(ps), 7):
        r = shg.solve(ps[i])
        assert np.array_equal(sigs[i].cpu().numpy(), r.signal), i
        assert np.array_equal(pumps[i].cpu().numpy(), r.pump), i
        assert abs(power[i] - r.sh_power) <= 1e-12 * abs(r.sh_power), i


def test_batch_fp64_matches_oracle():
    ps = sweep(64, 12, seed=3)
    pumps, sigs = device_outputs(ps)
    power = shg.solve_batch_device(ps, pumps, sigs)
    for i, p in enumerate(ps):
        rc, pump, sig, st, _ = O.solve(p)
        assert rc == 0
        got = sigs[i].cpu().numpy()
        assert np.linalg.norm(got - sig) / np.linalg.norm(sig) <= 1e-10, i
        assert abs(power[i] - st.sh_power) <= 1e-12 * st.sh_power, i


@pytest.mark.parametrize("precision", [64, 32])
def test_plan_replays_equal_direct_batch(precision):
    import torch
    ps = sweep(precision, 40, seed=10 + precision)
    ref_p, ref_s = device_outputs(ps)
    ref_power = shg.solve_batch_device(ps, ref_p, ref_s)
    pumps, sigs = device_outputs(ps)
    plan = shg.BatchPlan(ps, pumps, sigs)
    try:
        for replay in range(3):
            for t in sigs:
                t.fill_(float("nan"))
            torch.cuda.synchronize()
            plan.launch()
            power = plan.powers()
            for i in range(len(ps)):
                assert torch.equal(sigs[i], ref_s[i]), (replay, i)
                assert torch.equal(pumps[i], ref_p[i]), (replay, i)
            assert np.array_equal(power, ref_power), replay
    finally:
        plan.close()


def test_plan_rejects_bad_input():
    with pytest.raises(shg.ShgError) as e:
        shg.BatchPlan([P.config_plain_64().replace(nx=50, ny=50)])
    assert e.value.status in (P.SHG_ERR_UNSUPPORTED, P.SHG_ERR_INVALID)
    with pytest.raises(shg.ShgError):
        shg.BatchPlan([P.config_plain_64(), P.config_plain_64().replace(precision=32)])


@pytest.fixture
def default_schedules():
    """The tuners' choices hold for the process: put the compiled defaults back afterwards."""
    yield
    shg.autotune_reset()


@pytest.mark.parametrize("precision,n", [(32, 128), (32, 256), (64, 128)])
def test_autotune_keeps_results(precision, n, default_schedules):
    """The tuner times every compiled split of the class and keeps the fastest; the fields
    of the class are the same bits before and after, the SH power agrees to rounding."""
    import torch
    ps = [p for p in sweep(precision, 60, seed=n + precision) if p.nx == n][:6]
    if not ps:
        ps = [P.workload(n, 9, 4000.0, 5.0, 30.0, 2000.0, 30.0, precision=precision)]
    before_p, before_s = device_outputs(ps)
    pw0 = shg.solve_batch_device(ps, before_p, before_s)
    r = shg.autotune(precision, n)
    assert r["n"] == n and r["precision"] == precision and r["candidates"] >= 1
    assert r["pt_steps_per_s"] >= r["default_pt_steps_per_s"] > 0
    after_p, after_s = device_outputs(ps)
    pw1 = shg.solve_batch_device(ps, after_p, after_s)
    torch.cuda.synchronize()
    for i in range(len(ps)):
        assert torch.equal(before_s[i], after_s[i]) and torch.equal(before_p[i], after_p[i]), i
    assert np.allclose(pw0, pw1, rtol=1e-12 if precision == 64 else 1e-6, atol=0)


@pytest.mark.parametrize("precision", [32, 64])
def test_batch_autotune_keeps_results(precision, default_schedules):
    """The batch tuner scores each class's compiled variants by the time of the whole batch and
    keeps a change only when the batch gets faster.  The fields agree with the default
    schedule's to the multi-pass-against-fused tolerances (FP64 relative L2 <= 1e-13, FP32
    <= 1e-5): a fused split gives the same bits, the multi-pass march (a candidate at 256 x
    256) differs where the compiler contracts multiply-adds differently."""
    import torch
    ps = sweep(precision, 24, seed=7 + precision)
    before_p, before_s = device_outputs(ps)
    pw0 = shg.solve_batch_device(ps, before_p, before_s)
    res = shg.autotune_batch(ps)
    assert sorted(r["n"] for r in res) == sorted({p.nx for p in ps})
    for r in res:
        assert r["precision"] == precision and r["candidates"] >= 1
        assert r["pt_steps_per_s"] >= r["default_pt_steps_per_s"] > 0
    after_p, after_s = device_outputs(ps)
    pw1 = shg.solve_batch_device(ps, after_p, after_s)
    torch.cuda.synchronize()
    tol = 1e-13 if precision == 64 else 1e-5
    rel = lambda a, b: float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))
    for i in range(len(ps)):
        assert rel(after_s[i], before_s[i]) <= tol and rel(after_p[i], before_p[i]) <= tol, i
    assert np.allclose(pw0, pw1, rtol=1e-12 if precision == 64 else 1e-5, atol=0)
    with pytest.raises(shg.ShgError) as e:
        shg.autotune_batch([ps[0].replace(march=P.SHG_MARCH_FUSED)])
    assert e.value.status == P.SHG_ERR_INVALID


@pytest.mark.parametrize("cluster,threads", [(8, 256), (16, 512)])
def test_pinned_schedule_gives_the_same_fields(cluster, threads, default_schedules):
    """shg_set_schedule picks a compiled 256 x 256 split without timing; the per-point
    arithmetic is the split's, so the fields are the same bits as with the default split."""
    import torch
    ps = [P.workload(256, 9, 4000.0, 5.0 + i, 30.0, 2000.0, 30.0, precision=32) for i in range(5)]
    ref_p, ref_s = device_outputs(ps)
    shg.solve_batch_device(ps, ref_p, ref_s)
    shg.set_schedule(32, 256, cluster, threads)
    got_p, got_s = device_outputs(ps)
    shg.solve_batch_device(ps, got_p, got_s)
    torch.cuda.synchronize()
    for i in range(len(ps)):
        assert torch.equal(got_s[i], ref_s[i]) and torch.equal(got_p[i], ref_p[i]), i


def test_autotune_rejects_unbuilt_class():
    with pytest.raises(shg.ShgError) as e:
        shg.autotune(32, 100)
    assert e.value.status == P.SHG_ERR_UNSUPPORTED


def test_host_buffer_batch_equals_device_batch():
    import torch
    ps = sweep(64, 9, seed=21)
    pumps, sigs, power = shg.solve_batch(ps)
    dp, ds = device_outputs(ps)
    pw = shg.solve_batch_device(ps, dp, ds)
    torch.cuda.synchronize()
    assert np.array_equal(power, pw)
    for i in range(len(ps)):
        assert np.array_equal(sigs[i], ds[i].cpu().numpy()) and np.array_equal(pumps[i], dp[i].cpu().numpy())


@pytest.mark.parametrize("precision", [32, 64])
def test_pinned_host_outputs_written_by_the_march(precision):
    """Page-locked host outputs are written by the march through their device mapping, with no
    staging copy; a batch that mixes them with pageable arrays and missing outputs, and holds
    a 512 x 512 instance (multi-pass march), still equals the device batch bit for bit."""
    import torch
    ps = sweep(precision, 7, seed=33) + [P.workload(512, 5, 4000.0, 10.0, 30.0, 2000.0, 30.0, precision=precision)]
    dt = torch.complex128 if precision == 64 else torch.complex64
    npdt = np.complex128 if precision == 64 else np.complex64
    pumps, sigs = [], []
    for i, p in enumerate(ps):
        kind = i % 3  # 0: pinned, 1: pageable numpy, 2: pinned pump only
        if kind == 1:
            pumps.append(np.full((p.ny, p.nx), np.nan, dtype=npdt))
            sigs.append(np.full((p.ny, p.nx), np.nan, dtype=npdt))
        else:
            pumps.append(torch.full((p.ny, p.nx), float("nan"), dtype=dt).pin_memory())
            sigs.append(None if kind == 2 else torch.full((p.ny, p.nx), float("nan"), dtype=dt).pin_memory())
    _, _, power = shg.solve_batch(ps, pumps, sigs)
    dp, ds = device_outputs(ps)
    pw = shg.solve_batch_device(ps, dp, ds)
    torch.cuda.synchronize()
    assert np.array_equal(power, pw)
    as_np = lambda a: a if isinstance(a, np.ndarray) else a.numpy()
    for i in range(len(ps)):
        assert np.array_equal(as_np(pumps[i]), dp[i].cpu().numpy()), i
        if sigs[i] is not None:
            assert np.array_equal(as_np(sigs[i]), ds[i].cpu().numpy()), i
