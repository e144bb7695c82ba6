"""Calls from several host threads at once (each call on its own stream, the last error kept
per thread): results equal the same calls made one after the other, bit for bit.  The
allocation-free batch entry point is excluded: it shares one static scratch array and is
documented as not safe to overlap."""
import concurrent.futures as cf

import numpy as np
import pytest

from cushg_b200 import params as P
from cushg_b200 import shg

pytestmark = pytest.mark.gpu


def thermal_case(i):
    p = P.workload(64, 12, 6000.0, 20.0, 30.0, 3000.0, 30.0 + 3.0 * i, precision=64, thermal=1)
    p.alpha_p, p.alpha_s, p.beta_s = 2e-5, 1e-4, 1e-3
    p.max_outer = 2
    p.check_every = 50
    p.conv_rule = P.SHG_CONV_MAXABS
    p.jacobi_tol = 1e-3
    return p


def test_thermal_solves_from_threads_equal_sequential():
    ps = [thermal_case(i) for i in range(4)]
    seq = [shg.solve(p, want_temperature=True) for p in ps]
    with cf.ThreadPoolExecutor(max_workers=4) as ex:
        par = list(ex.map(lambda p: shg.solve(p, want_temperature=True), ps))
    for a, b in zip(seq, par):
        assert np.array_equal(a.signal, b.signal) and np.array_equal(a.pump, b.pump)
        assert np.array_equal(a.temperature, b.temperature)
        assert a.stats.jacobi_sweeps == b.stats.jacobi_sweeps


def test_thermal_grads_and_batches_from_threads():
    tg = []
    for i in range(2):
        p = P.workload(256, 9, 4000.0, 30.0, 25.0, 2000.0, 34.0 + i, precision=32, thermal=1)
        p.alpha_p = p.alpha_s = p.beta_s = 0.0
        p.conv_rule = P.SHG_CONV_FIXED
        p.max_sweeps, p.max_outer = 40, 1
        tg.append(p)
    batch = [P.workload(n, 10, 4000.0, 10.0, 25.0, 2000.0, 30.0, precision=32) for n in (64, 128, 192, 256) * 3]
    seq_g = [shg.thermal_grad(p) for p in tg]
    seq_b = shg.solve_batch(batch)
    with cf.ThreadPoolExecutor(max_workers=4) as ex:
        fg = [ex.submit(shg.thermal_grad, p) for p in tg]
        fb = [ex.submit(shg.solve_batch, batch) for _ in range(2)]
        par_g = [f.result() for f in fg]
        par_b = [f.result() for f in fb]
    for a, b in zip(seq_g, par_g):
        assert a["d_temp"] == b["d_temp"] and a["sh_power"] == b["sh_power"]
    for pumps, sigs, power in par_b:
        assert np.array_equal(power, seq_b[2])
        for i in range(len(batch)):
            assert np.array_equal(sigs[i], seq_b[1][i]) and np.array_equal(pumps[i], seq_b[0][i])


def test_errors_stay_on_their_thread():
    bad = P.config_plain_64().replace(nx=50, ny=50)
    good = P.config_plain_64()

    def run(p):
        try:
            shg.solve(p)
            return ""
        except shg.ShgError as e:
            return str(e)

    with cf.ThreadPoolExecutor(max_workers=8) as ex:
        futs = [ex.submit(run, bad if i % 2 == 0 else good) for i in range(8)]
        out = [f.result() for f in futs]
    for i, msg in enumerate(out):
        assert ("grid side 50" in msg) if i % 2 == 0 else msg == "", (i, msg)
