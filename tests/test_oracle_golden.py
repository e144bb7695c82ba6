"""Pin the CPU oracle against the reference's own outputs.

The fixtures in tests/golden/ were produced by running the reference program
(alfredos84/cuSHG, patched to FP64 and to each case's constants by oracle/ref_build.py)
on a B200 with oracle/make_golden.py.  The reference has no tests or golden vectors of
its own, so these runs are what pins the oracle.
"""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN
from cushg_b200 import params as P
from oracle import golden_cases as G
from oracle import oracle as O

FP64_CASES = [n for n, c in G.CASES.items() if c["precision"] == 64]


def load(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    return z, json.loads(str(z["meta"]))


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("name", FP64_CASES)
def test_oracle_matches_reference_fp64(name):
    z, meta = load(name)
    p = G.params_of(name)
    # the fixture was made from exactly these parameters (fields added to shg_params after
    # the fixture was written are execution settings at their defaults)
    d = p.as_dict()
    assert {k: v for k, v in d.items() if k in meta["params"]} == meta["params"]
    assert all(d[k] == 0 for k in d if k not in meta["params"])
    rc, pump, sig, st, T = O.solve(p, want_temperature=True)
    assert rc == 0
    # output-field relative L2 <= 1e-10 for the plain FP64 path
    assert rel_l2(pump, z["pump"]) < 1e-10
    assert rel_l2(sig, z["signal"]) < 1e-10
    if p.thermal:
        assert st.jacobi_sweeps == sum(meta["jacobi_sweeps"])
        assert st.outer_iterations == len(meta["jacobi_sweeps"])
        assert np.abs(T - z["T"]).max() < 1e-9
    else:
        ref_power = P.sh_power_of(p, z["signal"])
        # SH power relative error <= 1e-12
        assert abs(st.sh_power - ref_power) / ref_power < 1e-12


def test_oracle_fp32_close_to_reference_fp32():
    """The float build of the reference against the float oracle: same arithmetic up to
    FFT and FMA rounding, so they agree at float noise level."""
    z, meta = load("plain32_c1")
    p = G.params_of("plain32_c1")
    rc, pump, sig, st, _ = O.solve(p)
    assert rc == 0
    assert rel_l2(pump, z["pump"]) < 1e-4
    assert rel_l2(sig, z["signal"]) < 1e-3


def test_reference_fp32_error_vs_fp64():
    """How far the reference's own float build is from its FP64 build at the same inputs
    (recorded: the reference's FP32 error is dominated by the float Δk cancellation)."""
    z32, _ = load("plain32_c1")
    z64, _ = load("plain64_c1")
    e = rel_l2(z32["signal"], z64["signal"])
    assert 1e-6 < e < 1e-1


@pytest.mark.parametrize("waist_y", [0.0, 45.0, 20.0])
def test_initial_pump_carries_the_pump_power(waist_y):
    """setPump's normalisation (Efields.h:99): the z = 0 pump carries the pump power, for the
    round beam and for the elliptical variant (normalised with waist * waist_y)."""
    p = P.workload(128, 12, 8000.0, 10.0, 30.0, 2000.0, 30.0, precision=64).replace(waist_y=waist_y)
    p.lx = p.ly = 12 * max(p.waist, waist_y)
    pump = O.set_pump(p, p.temp).reshape(p.ny, p.nx)
    n = P.sellmeier(p.lambda_p, p.temp)
    dx, dy = p.lx / (p.nx - 1), p.ly / (p.ny - 1)
    power = 0.5 * P.EPS0 * P.C_UM_PS * n * float(np.sum(np.abs(pump) ** 2)) * dx * dy
    assert abs(power - p.power) <= 1e-9 * p.power
