"""The crystal selector (shg_params.crystal): MgO:sPPLT, the reference's only crystal
(src/headers/Crystal.h:54-70), and 5 mol% MgO:PPLN, which the reference's README.md:52 names
but its headers do not carry.  MgO:PPLN uses the temperature-dependent Sellmeier equation of
Gayer et al., Appl. Phys. B 91, 343 (2008), and lithium niobate's thermal expansion of the
grating (α = 1.54e-5, β = 5.3e-9).

No reference output exists for MgO:PPLN, so its index is pinned in two ways. The oracle's C
function is compared with an independent Python restatement of the published equation. The
first-order QPM period it gives for 1064 -> 532 nm SHG lies in the 6.8-7.1 µm range of
commercial MgO:PPLN gratings for that process."""
import ctypes
import math

import pytest

from cushg_b200 import params as P
from cushg_b200 import shg
from oracle import oracle as O


def gayer_ne(lam, t):
    # the published form, written out term by term
    f = (t - 24.5) * (t + 570.82)
    a = [5.756, 0.0983, 0.2020, 189.32, 12.52, 1.32e-2]
    b = [2.860e-6, 4.700e-8, 6.113e-8, 1.516e-4]
    n2 = (a[0] + b[0] * f + (a[1] + b[1] * f) / (lam ** 2 - (a[2] + b[2] * f) ** 2)
          + (a[3] + b[3] * f) / (lam ** 2 - a[4] ** 2) - a[5] * lam ** 2)
    return math.sqrt(n2)


@pytest.mark.parametrize("lam", [0.532, 0.775, 1.064, 1.55])
@pytest.mark.parametrize("t", [20.0, 40.0, 80.0, 150.0])
def test_ppln_index_matches_published_equation(lam, t):
    n_oracle = O.sellmeier(lam, t, P.SHG_CRYSTAL_MGO_PPLN)
    assert abs(n_oracle - gayer_ne(lam, t)) <= 1e-14
    assert abs(P.sellmeier(lam, t, P.SHG_CRYSTAL_MGO_PPLN) - n_oracle) <= 1e-14
    # the default crystal is still sPPLT, and the two indices differ
    assert O.sellmeier(lam, t) == O.sellmeier(lam, t, P.SHG_CRYSTAL_MGO_SPPLT)
    assert abs(O.sellmeier(lam, t) - n_oracle) > 1e-3


def test_ppln_known_values():
    # n_e of MgO:LN at 1064 nm near room temperature is about 2.148, at 532 nm about 2.22-2.23
    assert 2.14 < P.sellmeier(1.064, 25.0, P.SHG_CRYSTAL_MGO_PPLN) < 2.155
    assert 2.215 < P.sellmeier(0.532, 25.0, P.SHG_CRYSTAL_MGO_PPLN) < 2.235
    # the index rises with temperature
    assert P.sellmeier(1.064, 80.0, 1) > P.sellmeier(1.064, 25.0, 1)
    # first-order QPM period of 1064 -> 532 nm SHG
    for t in (25.0, 40.0, 80.0):
        assert 6.8 < P.qpm_period(t, 1.064, P.SHG_CRYSTAL_MGO_PPLN) < 7.1
    # and the sPPLT period of the reference's configuration stays where it was
    assert 7.9 < P.qpm_period(25.0) < 8.1


def test_ppln_phase_matched_at_its_qpm_temperature():
    p = P.workload(64, 12, 10000.0, 5.0, 30.0, 5000.0, 40.0, precision=64)
    p.crystal = P.SHG_CRYSTAL_MGO_PPLN
    p.period = P.qpm_period(40.0, p.lambda_p, P.SHG_CRYSTAL_MGO_PPLN)
    assert abs(O.delta_k(p, 40.0)) < 1e-10
    assert abs(O.delta_k(p, 45.0)) > 1e-5
    # with the sPPLT index the same grating is far from phase matching
    q = p.replace(crystal=P.SHG_CRYSTAL_MGO_SPPLT)
    assert abs(O.delta_k(q, 40.0)) > 0.1


def test_check_params_accepts_both_crystals_only():
    L = shg.lib()
    p = P.workload(64, 12, 10000.0, 5.0, 30.0, 5000.0, 40.0, precision=64)
    for c in (P.SHG_CRYSTAL_MGO_SPPLT, P.SHG_CRYSTAL_MGO_PPLN):
        assert L.shg_check_params(ctypes.byref(p.replace(crystal=c))) == P.SHG_OK
    for c in (2, -1):
        assert L.shg_check_params(ctypes.byref(p.replace(crystal=c))) == P.SHG_ERR_UNSUPPORTED
