"""The second crystal, 5 mol% MgO:PPLN (shg_params.crystal = SHG_CRYSTAL_MGO_PPLN), through
every path whose constants depend on the crystal, against the oracle:

* the plain march: fused at 64 and 256, multi-pass at 512, FP64;
* FP32 against the FP64 oracle;
* the thermal run, whose per-voxel n(T) and Δk(T) are computed on the device;
* the adjoint's temperature derivative, which uses dn/dT;
* the forward-mode dJ/dT_oven, which uses the per-voxel optics tangents.

Tolerances are those of the sPPLT tests: FP64 fields 1e-10 relative L2, SH power 1e-12 (plain)
and 1e-10 (thermal); FP32 SH power 1e-5 of FP64; the adjoint within 1e-5 of central
differences; the thermal tangent within 1e-6 of central differences without absorption."""
import numpy as np
import pytest

from cushg_b200 import params as P
from cushg_b200 import shg
from oracle import oracle as O

pytestmark = pytest.mark.gpu

LN = P.SHG_CRYSTAL_MGO_PPLN


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a, np.complex128) - b) / np.linalg.norm(b))


def ppln(n, nz, temp=40.0, precision=64, thermal=0, lz=8000.0, waist=25.0):
    p = P.workload(n, nz, lz, 20.0, waist, 0.45 * lz, temp, precision=precision, thermal=thermal)
    p.crystal = LN
    p.period = P.qpm_period(temp + 0.3, p.lambda_p, LN)  # near, not at, phase matching
    return p


@pytest.mark.parametrize("n", [64, 256, 512])
def test_ppln_plain_matches_oracle(n):
    p = ppln(n, 9 if n == 512 else 14)
    r = shg.solve(p)
    rc, pump, sig, st, _ = O.solve(p)
    assert rc == 0
    assert rel_l2(r.pump, pump) <= 1e-10 and rel_l2(r.signal, sig) <= 1e-10
    assert abs(r.sh_power - st.sh_power) <= 1e-12 * st.sh_power
    # the crystal matters: the same run with sPPLT constants differs
    other = shg.solve(p.replace(crystal=P.SHG_CRYSTAL_MGO_SPPLT))
    assert abs(other.sh_power - r.sh_power) > 1e-3 * r.sh_power


@pytest.mark.parametrize("n", [128, 256])
def test_ppln_fp32_against_fp64_oracle(n):
    p = ppln(n, 40)
    rc, pump, sig, st, _ = O.solve(p)
    r = shg.solve(p.replace(precision=32))
    assert rel_l2(r.signal, sig) <= 1e-4
    assert abs(r.sh_power - st.sh_power) / st.sh_power <= 1e-5


def test_ppln_thermal_matches_oracle():
    p = ppln(64, 12, temp=45.0, thermal=1, lz=6000.0)
    p.alpha_p, p.alpha_s, p.beta_s = 2e-5, 1e-4, 1e-3
    p.max_outer = 2
    p.check_every = 200
    p.conv_rule = P.SHG_CONV_MAXABS
    p.jacobi_tol = 1e-3
    r = shg.solve(p, want_temperature=True)
    rc, pump, sig, st, T = O.solve(p, want_temperature=True)
    assert rc == 0
    assert r.stats.jacobi_sweeps == st.jacobi_sweeps
    assert np.abs(r.temperature - T).max() <= 1e-9
    assert rel_l2(r.signal, sig) <= 1e-10
    assert abs(r.sh_power - st.sh_power) / st.sh_power <= 1e-10


def test_ppln_adjoint_temperature_derivative():
    p = ppln(64, 31)
    g = shg.grad(p)
    h = 1e-4
    d = (shg.sh_power(p.replace(temp=p.temp + h, t_peltier=p.temp + h))
         - shg.sh_power(p.replace(temp=p.temp - h, t_peltier=p.temp - h))) / (2 * h)
    assert abs(g["d_temp"] - d) <= 1e-5 * abs(d), (g["d_temp"], d)


def test_ppln_thermal_grad_matches_finite_differences():
    p = ppln(256, 9, temp=34.0, thermal=1, lz=4000.0)
    p.t_peltier = p.temp
    p.alpha_p = p.alpha_s = p.beta_s = 0.0
    p.conv_rule = P.SHG_CONV_FIXED
    p.max_sweeps = 60
    p.max_outer = 1
    g = shg.thermal_grad(p)
    h = 1e-3
    jp = shg.solve(p.replace(temp=p.temp + h, t_peltier=p.t_peltier + h)).sh_power
    jm = shg.solve(p.replace(temp=p.temp - h, t_peltier=p.t_peltier - h)).sh_power
    d = (jp - jm) / (2 * h)
    assert abs(g["d_temp"] - d) <= 1e-6 * abs(d), (g["d_temp"], d)
