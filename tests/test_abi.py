"""C-ABI checks that need no GPU: the library loads, exports every entry point that
include/shg.h declares, and validates parameters like the reference's constraints."""
import ctypes
import os
import re

import pytest

from conftest import ROOT
from cushg_b200 import params as P
from cushg_b200 import shg


def declared_entry_points():
    text = open(os.path.join(ROOT, "include", "shg.h")).read()
    return sorted(set(re.findall(r"SHG_API\s+[\w\s\*]+?\b(shg_\w+)\s*\(", text)))


def test_header_and_binding_agree():
    assert sorted(shg.EXPORTS) == declared_entry_points()


def test_library_exports_every_declared_symbol():
    L = shg.lib()
    for name in declared_entry_points():
        assert hasattr(L, name), name


def test_default_params_are_the_reference_configuration():
    d = shg.default_params()
    r = P.reference_defaults()
    assert d.as_dict() == r.as_dict()
    assert (d.nx, d.ny, d.nz) == (128, 128, 100)          # src/cuSHG.cu:11-13
    assert (d.lx, d.ly, d.lz) == (2000.0, 1000.0, 30000.0)  # Crystal.h:31-33
    assert d.focus == 0.5 * d.lz                            # cuSHG.cu:48


def test_steps_follow_the_output_slice_rule():
    p = P.config_plain_64()
    assert shg.steps(p) == p.nz - 1
    assert shg.steps(p.replace(thermal=1)) == p.nz


@pytest.mark.parametrize("field,value", [
    ("nx", 63), ("nz", 1), ("precision", 16), ("waist", 0.0), ("lx", -1.0), ("alpha_p", -1e-6),
    ("power", float("nan")), ("lambda_p", 0.0), ("fp32_guard", -1e-5), ("fp32_guard", float("inf")),
])
def test_invalid_params_are_rejected(field, value):
    p = P.config_plain_64().replace(**{field: value})
    assert shg.check_params(p) == P.SHG_ERR_INVALID
    assert shg.last_error() != ""


def test_unbuilt_grid_is_unsupported():
    p = P.config_plain_64().replace(nx=100, ny=100)
    assert shg.check_params(p) == P.SHG_ERR_UNSUPPORTED


def test_valid_params_pass():
    for p in [P.config_plain_64(), P.config_thermal_128(), *P.config_sweep(16)]:
        assert shg.check_params(p) == P.SHG_OK, shg.last_error()


def test_solve_without_device_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(shg.ShgError) as e:
        shg.solve(P.config_plain_64())
    assert e.value.status == P.SHG_ERR_NO_DEVICE


def test_status_strings():
    L = shg.lib()
    assert L.shg_status_string(0) == b"ok"
    assert L.shg_version().startswith(b"libshg_b200")


def test_march_selector_is_validated():
    """512 x 512 is built as a multi-pass march only, 64 x 64 as a fused march only."""
    p512 = P.workload(512, 9, 6000.0, 5.0, 30.0, 3000.0, 30.0, precision=32)
    assert shg.check_params(p512) == P.SHG_OK
    assert shg.check_params(p512.replace(march=P.SHG_MARCH_MULTIPASS)) == P.SHG_OK
    assert shg.check_params(p512.replace(march=P.SHG_MARCH_FUSED)) == P.SHG_ERR_UNSUPPORTED
    assert shg.check_params(p512.replace(march=7)) == P.SHG_ERR_INVALID
    p64 = P.config_plain_64()
    assert shg.check_params(p64.replace(march=P.SHG_MARCH_MULTIPASS)) == P.SHG_ERR_UNSUPPORTED
    assert shg.check_params(p64.replace(march=P.SHG_MARCH_FUSED)) == P.SHG_OK


@pytest.mark.parametrize("n,fused,multipass", [(64, True, False), (128, True, True), (256, True, True),
                                               (512, False, True)])
def test_thermal_marches_built_per_side(n, fused, multipass):
    """Thermal runs: fused cluster marches for sides up to 256, multi-pass marches at 128, 256
    and 512 (the automatic choice where built); a side with neither is unsupported."""
    p = P.workload(n, 9, 6000.0, 5.0, 30.0, 3000.0, 30.0, precision=64, thermal=1)
    ok = lambda built: P.SHG_OK if built else P.SHG_ERR_UNSUPPORTED  # noqa: E731
    assert shg.check_params(p.replace(march=P.SHG_MARCH_FUSED)) == ok(fused)
    assert shg.check_params(p.replace(march=P.SHG_MARCH_MULTIPASS)) == ok(multipass)
    assert shg.check_params(p) == P.SHG_OK


def test_fixed_sweep_rule_needs_counts():
    p = P.config_thermal_128().replace(conv_rule=P.SHG_CONV_FIXED, max_sweeps=0)
    assert shg.check_params(p) == P.SHG_ERR_INVALID
    assert shg.check_params(p.replace(max_sweeps=10, max_outer=2)) == P.SHG_OK
    assert shg.check_params(p.replace(conv_rule=3)) == P.SHG_ERR_INVALID


def test_batch_autotune_arguments_are_checked_before_the_device():
    """shg_autotune_batch validates its arguments on the host: a null or empty batch, a null
    result array, a forced march and mixed precisions are SHG_ERR_INVALID; a valid batch on a
    machine without a GPU is SHG_ERR_NO_DEVICE.  shg_autotune_reset never fails."""
    import ctypes
    from cushg_b200.shg import ShgTuneResult, ShgParams

    L = shg.lib()
    p = P.config_plain_64().replace(precision=32)
    out = (ShgTuneResult * 4)()
    n = ctypes.c_int32(0)

    def call(ps, count, res=out, cap=4):
        arr = (ShgParams * max(1, len(ps)))(*ps) if ps else None
        return L.shg_autotune_batch(arr, count, res, cap, ctypes.byref(n))

    assert call([], 0) == P.SHG_ERR_INVALID
    assert call([p], 1, res=None) == P.SHG_ERR_INVALID
    assert call([p], 1, cap=0) == P.SHG_ERR_INVALID
    assert call([p.replace(march=P.SHG_MARCH_FUSED)], 1) == P.SHG_ERR_INVALID
    assert call([p, p.replace(precision=64)], 2) == P.SHG_ERR_INVALID
    import torch
    if not torch.cuda.is_available():
        assert call([p], 1) == P.SHG_ERR_NO_DEVICE
    L.shg_autotune_reset()


def test_set_schedule_finds_compiled_splits_only():
    """shg_set_schedule looks the split up among the compiled variants (no device needed)."""
    L = shg.lib()
    assert L.shg_set_schedule(32, 256, 8, 256) == P.SHG_OK
    assert L.shg_set_schedule(32, 256, 3, 256) == P.SHG_ERR_UNSUPPORTED
    assert L.shg_set_schedule(32, 100, 1, 128) == P.SHG_ERR_UNSUPPORTED
    assert L.shg_set_schedule(16, 256, 8, 256) == P.SHG_ERR_INVALID
    L.shg_autotune_reset()


def test_reserve_device_memory_checks_its_argument():
    import torch
    L = shg.lib()
    assert L.shg_reserve_device_memory(-1) == P.SHG_ERR_INVALID
    if not torch.cuda.is_available():
        assert L.shg_reserve_device_memory(1 << 20) == P.SHG_ERR_NO_DEVICE


def test_fp32_error_estimate_follows_the_phase_mismatch_cancellation():
    """shg_fp32_error_estimate is host arithmetic: the phase-matched run is well conditioned
    (the SH grows monotonically, the estimate is K sqrt(steps) times about 1), a run far from
    phase matching is worse, and more steps raise it as sqrt(steps)."""
    p = P.workload(128, 201, 10000.0, 10.0, 30.0, 5000.0, P.QPM_TEMP, precision=32)
    matched = shg.fp32_error_estimate(p)
    assert 0 < matched < 3 * 1.3e-7 * (p.nz - 1) ** 0.5
    far = shg.fp32_error_estimate(p.replace(temp=60.0, t_peltier=60.0))
    assert far > 3 * matched
    longer = shg.fp32_error_estimate(p.replace(nz=801))
    assert abs(longer / matched - 2.0) < 1e-6
    # an elliptical beam goes through the general envelope
    assert shg.fp32_error_estimate(p.replace(waist_y=45.0)) > 0
