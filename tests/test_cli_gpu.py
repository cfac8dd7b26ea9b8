"""The native drop-in CLI (bfpn_gpu_b200/bin/bfp_solver) end to end on the GPU:
the reference's output files (idd_output.txt, dose_output.txt,
energy_moments.txt, spot planes), their formats, and their values against the
oracle."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, table_dir
from bfpn_gpu_b200 import parse_args, read_tables
from oracle import oracle as O

pytestmark = pytest.mark.gpu

CLI = os.path.join(ROOT, "bfpn_gpu_b200", "bin", "bfp_solver")


def run_cli(tmp_path, args):
    r = subprocess.run([CLI] + args, cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr + r.stdout
    return r.stdout


def test_cli_outputs_match_oracle(tmp_path):
    args = ("60 --time 1.5 --data %s --lg 59 --ng 40 --energy 40 --sigma-e 2 --sigma-yz 0.4 --ny 6 --nz 5 "
            "--nmu 4 --nom 5 --ly 2 --lz 1.5 --lu 1 --lv 1.2 --trapezoidal-yz --save-energy-moments "
            "--spot-depths 0.5,1.0 --spot-prefix %s" % (table_dir("synthetic500"), tmp_path / "spot")).split()
    out = run_cli(tmp_path, args)
    assert "Solver completed. Paper-style IDD saved to idd_output.txt" in out
    cfg = parse_args(args)
    n = cfg.max_steps()
    mu, sig = read_tables(table_dir("synthetic500"), cfg.ng)
    ora = O.Oracle(cfg.grid(), cfg.phys(), mu, sig)
    idd_o, prox_o, mom_o, planes = [], [], [], {}
    t = 0.0
    for k in range(n):
        a, b = ora.step(1)
        idd_o.append(a[0])
        prox_o.append(b[0])
        mom_o.append(ora.energy_moments())
        t += cfg.dt()
        for d in cfg.spot_depths:
            if d not in planes and t + 0.5 * cfg.dt() >= d:
                planes[d] = (t, ora.spot_plane())
    lines = open(tmp_path / "idd_output.txt").read().splitlines()
    assert lines[0] == "# x_cm value" and len(lines) == n + 1
    x = np.array([float(l.split()[0]) for l in lines[1:]])
    assert lines[1].split()[0] == "%.17g" % cfg.dt()
    np.testing.assert_allclose(x, (np.arange(n) + 1) * cfg.dt(), rtol=0, atol=1e-15)
    idd = np.array([float(l.split()[1]) for l in lines[1:]])
    assert np.abs(idd - idd_o).max() <= 1e-10 * np.abs(idd_o).max()
    prox = np.loadtxt(tmp_path / "dose_output.txt")[:, 1]
    assert np.abs(prox - prox_o).max() <= 1e-10 * np.abs(prox_o).max()
    mom = np.loadtxt(tmp_path / "energy_moments.txt")
    assert mom.shape == (n * cfg.ng, 5)
    mom_ref = np.concatenate([m.reshape(-1, 2) for m in mom_o])
    assert np.abs(mom[:, 3:] - mom_ref).max() <= 1e-5 * np.abs(mom_ref).max()  # printed with 6 digits
    for d, (tact, plane_ref) in planes.items():
        name = tmp_path / ("spot_req%.2f_x%.2f.txt" % (d, tact))
        assert name.exists(), sorted(os.listdir(tmp_path))
        rows = [l for l in open(name).read().splitlines() if l and not l.startswith("#")]
        vals = np.array([float(r.split()[2]) for r in rows])
        assert vals.shape == plane_ref.shape
        assert np.abs(vals - plane_ref).max() <= 1e-5 * np.abs(plane_ref).max()  # printed with 6 digits


def test_cli_mixed_precision_runs(tmp_path):
    args = ("40 --time 12 --data %s --lg 59 --ng 40 --energy 40 --sigma-e 2 --sigma-yz 0.4 --ny 6 --nz 5 "
            "--nmu 4 --nom 5 --ly 2 --lz 1.5 --precision mixed --profile-steps" % table_dir("synthetic500")).split()
    out = run_cli(tmp_path, args)
    assert "Step timing summary (12 steps)" in out
    n = parse_args(args).max_steps()
    idd = np.loadtxt(tmp_path / "idd_output.txt", ndmin=2)
    assert n == 12 and idd.shape == (n, 2) and np.all(np.isfinite(idd[:, 1])) and np.abs(idd[:, 1]).max() > 0


def test_cli_reports_missing_tables(tmp_path):
    r = subprocess.run([CLI, "10", "--time", "0.1", "--data", str(tmp_path / "nowhere"), "--ny", "2", "--nz", "2",
                        "--nmu", "2", "--nom", "2", "--ng", "10"], cwd=tmp_path, capture_output=True, text=True)
    assert r.returncode == 1 and "Error:" in r.stderr


def test_cli_lite_memory_matches_oracle(tmp_path):
    args = ("50 --time 2 --data %s --lg 59 --ng 40 --energy 40 --sigma-e 2 --sigma-yz 0.4 --ny 6 --nz 5 "
            "--nmu 4 --nom 5 --ly 2 --lz 1.5 --lite-memory --save-energy-moments" % table_dir("synthetic500")).split()
    out = run_cli(tmp_path, args)
    assert "Mode: lite-memory primary-only" in out
    cfg = parse_args(args)
    mu, sig = read_tables(table_dir("synthetic500"), cfg.ng)
    idd_o, prox_o = O.Oracle(cfg.grid(), cfg.phys(), mu, sig).step(cfg.max_steps())
    res = np.loadtxt(tmp_path / "idd_output.txt")
    assert np.abs(res[:, 1] - idd_o).max() <= 1e-10 * np.abs(idd_o).max()
    assert not np.any(np.loadtxt(tmp_path / "dose_output.txt")[:, 1])
    assert not (tmp_path / "energy_moments.txt").exists()  # the lite loop writes no moments
