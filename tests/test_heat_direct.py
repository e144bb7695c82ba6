"""The direct heat solve on the CPU: the one-dimensional operators' modes, and the separable
solve of the scaled system against the fixed point of the oracle's Jacobi sweep (which does
not use the separable form), for both boundary models of the reference (Tfield.h:93-240)."""
import numpy as np
import pytest

from cushg_b200 import params as P
from cushg_b200 import shg

import heat_ref as H


def operator(m, d, lo, hi, bi):
    M = (np.diag(np.full(m, 2.0)) - np.diag(np.ones(m - 1), 1) - np.diag(np.ones(m - 1), -1)) / d**2
    if lo:
        M[0, 0] = 2 * (1 + bi) / d**2
        if m > 1:
            M[0, 1] = -2 / d**2
    if hi:
        M[-1, -1] = 2 * (1 + bi) / d**2
        if m > 1:
            M[-1, -2] = -2 / d**2
    return M


@pytest.mark.parametrize("m,lo,hi,bi", [(1, 0, 0, 0.0), (2, 1, 1, 0.3), (7, 0, 1, 0.01), (64, 1, 1, 0.0),
                                        (127, 0, 1, 2.5e-4), (256, 1, 1, 1e-3), (510, 0, 0, 0.0)])
def test_operator_modes_diagonalise(m, lo, hi, bi):
    d = 1.7
    lam, F, G = shg.heat_operator_modes(m, d, lo, hi, bi)
    M = operator(m, d, lo, hi, bi)
    scale = np.abs(M).max()
    assert np.abs(F @ G - np.eye(m)).max() < 1e-12 * m
    assert np.abs(G @ np.diag(lam) @ F - M).max() < 1e-12 * scale * m
    assert np.all(lam > -1e-12 * scale)


def test_operator_modes_rejects_bad_input():
    with pytest.raises(shg.ShgError):
        shg.heat_operator_modes(0, 1.0, 0, 0, 0.0)
    with pytest.raises(shg.ShgError):
        shg.heat_operator_modes(4, -1.0, 0, 0, 0.0)
    with pytest.raises(shg.ShgError):
        shg.heat_operator_modes(4, 1.0, 1, 1, -0.1)


@pytest.mark.parametrize("boundary", [P.SHG_BOUNDARY_TOP_OPEN, P.SHG_BOUNDARY_OVEN_SURROUNDED])
@pytest.mark.parametrize("n,nz", [(6, 5), (8, 7)])
def test_separable_solve_is_the_jacobi_fixed_point(boundary, n, nz):
    p, T0, Q = H.small_case(n, nz, boundary)
    ref = H.fixed_point(p, T0, Q)
    got = H.separable_solve(p, T0, Q)
    assert np.abs(got - ref).max() < 1e-9
    # and it is a fixed point of the oracle's sweep
    assert np.abs(H.O.jacobi_sweep(p, got.copy(), Q) - got).max() < 1e-9
    # the heat source matters (the check is not of a flat field)
    assert np.ptp(ref) > 1.0


def test_heat_solver_is_validated():
    p = P.config_thermal_128()
    p.heat_solver = 2
    assert shg.check_params(p) == P.SHG_ERR_INVALID
    p.heat_solver = P.SHG_HEAT_DIRECT
    assert shg.check_params(p) == P.SHG_OK


@pytest.mark.parametrize("m,robin,bi", [(2, 1, 0.5), (8, 0, 0.0), (128, 1, 1.4e-6), (510, 0, 0.0), (512, 1, 1.4e-6)])
def test_symmetric_operator_modes_have_exact_parity(m, robin, bi):
    """An operator with the same kind of end at both sides: its modes come even first, then
    odd, each exactly symmetric or antisymmetric under i -> m-1-i (the folded transforms of
    the direct solve rely on it)."""
    lam, F, G = shg.heat_operator_modes(m, 1.17, robin, robin, bi)
    h = m // 2
    scale = np.abs(F).max()
    assert np.abs(F[:h] - F[:h, ::-1]).max() <= 1e-15 * scale
    assert np.abs(F[h:] + F[h:, ::-1]).max() <= 1e-15 * scale
    assert np.abs(G[:, :h] - G[::-1, :h]).max() <= 1e-15 * np.abs(G).max()
    assert np.abs(F @ G - np.eye(m)).max() < 1e-12 * m
