"""The allocation-free batched march, for callers that cannot allocate device memory while
they run (hosts that give all free memory to their own allocator, latency-bound loops,
plugin hosts that forbid it).

shg_solve_batch_device_noalloc keeps its scratch in a fixed array inside the library; this
test calls it through the C ABI twice in a row, with different instance sets, and checks each
call against the allocating entry point shg_solve_batch_device with the tolerances of the
other parity tests (the two run the same kernels, so the results are in fact identical).
This file is collected last so that a run stopping at its first failure has already run
every other test.
"""
import numpy as np
import pytest

from cushg_b200 import params as P
from cushg_b200 import shg

pytestmark = pytest.mark.gpu


def instances(precision, seed):
    rng = np.random.default_rng(seed)
    out = []
    for n in (64, 128, 32, 256, 96, 192):
        waist = float(rng.uniform(15, 40))
        lz = float(rng.choice([4000.0, 8000.0]))
        p = P.workload(n, int(rng.integers(5, 12)), lz, float(rng.uniform(2, 30)), waist,
                       float(rng.uniform(0, lz)), float(rng.uniform(25, 45)), precision=precision)
        out.append(p)
    return out


def outputs(ps):
    import torch
    dt = torch.complex128 if ps[0].precision == 64 else torch.complex64
    return ([torch.full((p.ny, p.nx), float("nan"), dtype=dt, device="cuda") for p in ps],
            [torch.full((p.ny, p.nx), float("nan"), dtype=dt, device="cuda") for p in ps])


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_noalloc_batch_matches_allocating_batch_on_two_calls_in_a_row():
    import torch
    for call, (precision, seed) in enumerate([(64, 1), (32, 2)]):
        ps = instances(precision, seed)
        ref_p, ref_s = outputs(ps)
        ref_power = shg.solve_batch_device(ps, ref_p, ref_s)
        got_p, got_s = outputs(ps)
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        got_power = shg.solve_batch_device_noalloc(ps, got_p, got_s)
        torch.cuda.synchronize()
        if call > 0:
            # after the first call's device set-up, a call takes no device memory
            assert torch.cuda.mem_get_info()[0] == free_before
        field_tol = 1e-10 if precision == 64 else 1e-5
        power_tol = 1e-12 if precision == 64 else 1e-5
        for i in range(len(ps)):
            a, b = got_s[i].cpu().numpy(), ref_s[i].cpu().numpy()
            assert np.isfinite(a).all(), (call, i)
            assert rel_l2(a, b) <= field_tol, (call, i)
            assert rel_l2(got_p[i].cpu().numpy(), ref_p[i].cpu().numpy()) <= field_tol, (call, i)
            assert abs(got_power[i] - ref_power[i]) <= power_tol * abs(ref_power[i]), (call, i)


def test_noalloc_rejects_more_instances_than_its_scratch_holds():
    ps = [P.config_plain_64().replace(nz=4)] * (shg.NOALLOC_MAX_INSTANCES + 1)
    with pytest.raises(shg.ShgError) as e:
        shg.solve_batch_device_noalloc(ps, None, None)
    assert e.value.status == P.SHG_ERR_INVALID
    assert "64" in str(e.value)
