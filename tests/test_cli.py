"""The command-line drop-in (cushg_b200/cushg) that replaces the reference program's main
(src/cuSHG.cu:27-113): same five positional arguments, the compile-time constants as
options, the reference's .dat files as output."""
import json
import os
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT
from cushg_b200 import params as P
from cushg_b200 import shg
from oracle import golden_cases as G
from oracle import oracle as O

CLI = os.path.join(ROOT, "cushg_b200", "cushg")


def read_matrix(path):
    rows = [[float(v) for v in line.strip().split("\t") if v] for line in open(path) if line.strip()]
    return np.asarray(rows)


def test_cli_usage_without_arguments():
    r = subprocess.run([CLI], capture_output=True, text=True)
    assert r.returncode == 2
    assert "usage" in r.stderr


def test_cli_rejects_an_unknown_crystal():
    r = subprocess.run([CLI, "5", "30", "40", "1", "0", "--crystal", "bbo"], capture_output=True, text=True)
    assert r.returncode == 2
    assert "--crystal takes spplt or ppln" in r.stderr


def cli_args(p, save_only_last=1, save_t=0):
    a = [CLI, repr(p.power), repr(p.waist), repr(p.temp), str(save_only_last), str(save_t),
         "--nx", str(p.nx), "--nz", str(p.nz), "--lx", repr(p.lx), "--ly", repr(p.ly), "--lz", repr(p.lz),
         "--focus", repr(p.focus), "--t-inf", repr(p.t_inf), "--deff", repr(p.deff), "--period", repr(p.period),
         "--alpha-p", repr(p.alpha_p), "--alpha-s", repr(p.alpha_s), "--beta-s", repr(p.beta_s),
         "--rho-p", repr(p.rho_p), "--rho-s", repr(p.rho_s), "--kappa", repr(p.kappa), "--h-conv", repr(p.h_conv),
         "--precision", str(p.precision)]
    if p.crystal == P.SHG_CRYSTAL_MGO_PPLN:
        a += ["--crystal", "ppln"]
    if p.thermal:
        a += ["--thermal", "--max-outer", str(p.max_outer), "--check-every", str(p.check_every)]
        if p.boundary == P.SHG_BOUNDARY_OVEN_SURROUNDED:
            a += ["--boundary", "oven-surrounded"]
    return a


@pytest.mark.gpu
def test_cli_reproduces_reference_output_files(tmp_path):
    name = "plain64_c1"
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    p = G.params_of(name)
    r = subprocess.run(cli_args(p), cwd=tmp_path, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    pump = read_matrix(tmp_path / "Pump_out_r.dat") + 1j * read_matrix(tmp_path / "Pump_out_i.dat")
    sig = read_matrix(tmp_path / "Signal_out_r.dat") + 1j * read_matrix(tmp_path / "Signal_out_i.dat")
    assert pump.shape == (p.ny, p.nx)
    assert np.linalg.norm(pump - z["pump"]) / np.linalg.norm(z["pump"]) <= 1e-10
    assert np.linalg.norm(sig - z["signal"]) / np.linalg.norm(z["signal"]) <= 1e-10
    assert list(tmp_path.glob("GPUTime_NZ_100_N_64_T.txt"))


@pytest.mark.gpu
def test_cli_thermal_with_temperature_dump(tmp_path):
    name = "thermal64_n32"
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    p = G.params_of(name)
    r = subprocess.run(cli_args(p, 1, 1), cwd=tmp_path, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    T = np.stack([read_matrix(tmp_path / f"Tfinal_{k}.dat") for k in range(p.nz)])
    # the reference writes temperatures at the stream's default 6 significant digits
    assert np.abs(T - z["T"]).max() <= 1e-3
    sig = read_matrix(tmp_path / "Signal_out_r.dat") + 1j * read_matrix(tmp_path / "Signal_out_i.dat")
    assert np.linalg.norm(sig - z["signal"]) / np.linalg.norm(z["signal"]) <= 1e-10


@pytest.mark.gpu
def test_slices_record_every_step():
    p = P.config_plain_64().replace(nz=9)
    pump_s, sig_s, st, _ = shg.solve_slices(p)
    last = shg.solve(p)
    assert np.array_equal(pump_s[-1], last.pump) and np.array_equal(sig_s[-1], last.signal)
    # plane 0 holds the initial fields, plane s the fields after s steps
    assert np.abs(sig_s[0]).max() == 0.0
    p0 = O.set_pump(p, p.temp)
    assert np.linalg.norm(pump_s[0] - p0) / np.linalg.norm(p0) <= 1e-13
    for s in (1, 4):
        a = p0.copy()
        b = np.zeros_like(a)
        O.march_plain(p, s, a, b)
        assert np.linalg.norm(sig_s[s] - b) / np.linalg.norm(b) <= 1e-10


@pytest.mark.gpu
def test_cli_every_slice_files(tmp_path):
    p = P.config_plain_64().replace(nz=6)
    r = subprocess.run(cli_args(p, save_only_last=0), cwd=tmp_path, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    pump_s, sig_s, _, _ = shg.solve_slices(p)
    for s in range(p.nz):
        sig = read_matrix(tmp_path / f"Signal_{s}_r.dat") + 1j * read_matrix(tmp_path / f"Signal_{s}_i.dat")
        assert np.allclose(sig, sig_s[s], rtol=0, atol=1e-18 + 1e-15 * np.abs(sig_s[s]).max())


@pytest.mark.gpu
def test_cli_sweep_mode_writes_the_script_folders(tmp_path):
    """cushg --sweep replaces src/cuSHG.sh: every (power, waist, temperature) combination runs
    (one batched call), and each run's Pump_out / Signal_out files land in the script's
    sPPLT_P_<P>_W_T1_<T>_WAIST_<W> folder, equal to the single run of that point."""
    base = P.workload(64, 12, 6000.0, 10.0, 25.0, 3000.0, 30.0, precision=64)
    extra = cli_args(base)[6:]  # every option, as for a single run
    r = subprocess.run([CLI, "--sweep", "10,20", "25", "30,35.5", "1", "0"] + extra, cwd=tmp_path,
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    for pw in ("10", "20"):
        for t in ("30", "35.5"):
            folder = tmp_path / f"sPPLT_P_{pw}_W_T1_{t}_WAIST_25"
            assert (folder / f"{folder.name}.txt").exists()
            p = base.replace(power=float(pw), temp=float(t), t_peltier=float(t))
            ref = shg.solve(p)
            got = read_matrix(folder / "Signal_out_r.dat") + 1j * read_matrix(folder / "Signal_out_i.dat")
            assert np.array_equal(got, ref.signal), (pw, t)
            gotp = read_matrix(folder / "Pump_out_r.dat") + 1j * read_matrix(folder / "Pump_out_i.dat")
            assert np.array_equal(gotp, ref.pump), (pw, t)


@pytest.mark.gpu
def test_cli_thermal_sweep_runs_as_one_batch(tmp_path):
    """A thermal sweep that keeps only the last slice runs its points as one shg_thermal_batch
    call (outer iterations in lockstep); every point's fields and temperature files equal the
    single run of that point, and the report says the run was batched."""
    base = P.workload(32, 12, 4000.0, 20.0, 25.0, 2000.0, 30.0, precision=64, thermal=1)
    base.alpha_p, base.alpha_s, base.beta_s = 2e-5, 1e-4, 1e-3
    base.max_outer = 2
    base.check_every = 500
    extra = cli_args(base)[6:]  # every option, as for a single run
    r = subprocess.run([CLI, "--sweep", "10,20", "25", "30,33", "1", "1"] + extra, cwd=tmp_path,
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert "batched thermal sweep of 4 runs" in r.stdout
    for pw in ("10", "20"):
        for t in ("30", "33"):
            folder = tmp_path / f"sPPLT_P_{pw}_W_T1_{t}_WAIST_25"
            p = base.replace(power=float(pw), temp=float(t), t_peltier=float(t))
            ref = shg.solve(p, want_temperature=True)
            got = read_matrix(folder / "Signal_out_r.dat") + 1j * read_matrix(folder / "Signal_out_i.dat")
            assert np.array_equal(got, ref.signal), (pw, t)
            gotp = read_matrix(folder / "Pump_out_r.dat") + 1j * read_matrix(folder / "Pump_out_i.dat")
            assert np.array_equal(gotp, ref.pump), (pw, t)
            for z in (0, p.nz - 1):  # Tfinal files: 6 significant digits, as the reference writes them
                assert np.allclose(read_matrix(folder / f"Tfinal_{z}.dat"), ref.temperature[z], rtol=1e-5, atol=0)


@pytest.mark.gpu
def test_cli_second_crystal_matches_the_library(tmp_path):
    """--crystal ppln selects MgO:PPLN: the .dat files hold the fields shg_solve gives for the
    same parameters (written at 20 significant digits)."""
    p = P.workload(64, 30, 8000.0, 20.0, 25.0, 3600.0, 40.0, precision=64)
    p.crystal = P.SHG_CRYSTAL_MGO_PPLN
    p.period = P.qpm_period(40.3, p.lambda_p, P.SHG_CRYSTAL_MGO_PPLN)
    r = subprocess.run(cli_args(p), cwd=tmp_path, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    sig = read_matrix(tmp_path / "Signal_out_r.dat") + 1j * read_matrix(tmp_path / "Signal_out_i.dat")
    ref = shg.solve(p).signal
    assert np.linalg.norm(sig - ref) / np.linalg.norm(ref) <= 1e-12
