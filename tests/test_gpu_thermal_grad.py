"""dJ/dT_oven of a thermal run through its temperature field (shg_thermal_grad), against
central finite differences of the whole thermal run.

The runs use a fixed sweep count, so both sides differentiate the same procedure.  The
forward-mode derivative carries the tangent of the heat source Q of every optical pass into
the next outer iteration's sweeps, so it is exact with absorption too: FP64 within 1e-6
relative of central differences without absorption (Q = 0), within 1e-4 with absorption and
two or three outer iterations, at 256 x 256 and 512 x 512; the FP32 derivative within 1e-3 of
FP64 central differences."""
import numpy as np
import pytest

from cushg_b200 import params as P
from cushg_b200 import shg

pytestmark = pytest.mark.gpu


def case(n=256, precision=64, absorb=False, outer=1, sweeps=60):
    p = P.workload(n, 9, 4000.0, 30.0, 25.0, 2000.0, 34.0, precision=precision, thermal=1)
    p.t_peltier = p.temp
    if absorb:
        p.alpha_p, p.alpha_s, p.beta_s = 2e-5, 1e-4, 1e-3
    else:
        p.alpha_p = p.alpha_s = p.beta_s = 0.0
    p.conv_rule = P.SHG_CONV_FIXED
    p.max_sweeps = sweeps
    p.max_outer = outer
    return p


def fd(p, h=1e-3):
    jp = shg.solve(p.replace(temp=p.temp + h, t_peltier=p.t_peltier + h)).sh_power
    jm = shg.solve(p.replace(temp=p.temp - h, t_peltier=p.t_peltier - h)).sh_power
    return (jp - jm) / (2 * h)


@pytest.mark.parametrize("n", [256, 512])
def test_thermal_grad_without_absorption_matches_finite_differences(n):
    p = case(n)
    g = shg.thermal_grad(p)
    ref = shg.solve(p)
    assert g["sh_power"] == ref.sh_power
    assert abs(g["sh_power_tangent_march"] - g["sh_power"]) <= 1e-11 * g["sh_power"]
    assert g["jacobi_sweeps"] == p.max_sweeps
    d = fd(p)
    assert abs(g["d_temp"] - d) <= 1e-6 * abs(d), (g["d_temp"], d)


@pytest.mark.parametrize("n,outer", [(256, 2), (256, 3), (512, 2)])
def test_thermal_grad_with_absorption_matches_finite_differences(n, outer):
    p = case(n, absorb=True, outer=outer)
    g = shg.thermal_grad(p)
    assert g["outer_iterations"] == outer
    assert g["sh_power"] == shg.solve(p).sh_power
    d = fd(p)
    assert abs(g["d_temp"] - d) <= 1e-4 * abs(d), (g["d_temp"], d)


@pytest.mark.parametrize("absorb", [False, True])
def test_thermal_grad_fp32_512(absorb):
    p = case(512, precision=32, absorb=absorb, outer=2 if absorb else 1)
    g = shg.thermal_grad(p)
    d = fd(p.replace(precision=64))
    assert abs(g["d_temp"] - d) <= 1e-3 * abs(d), (g["d_temp"], d)


def test_thermal_grad_rejects_unbuilt_sides():
    with pytest.raises(shg.ShgError) as e:
        shg.thermal_grad(case(128))
    assert e.value.status == P.SHG_ERR_UNSUPPORTED
