"""Parity against fixtures written by the reference's own CUDA solver.

tests/golden/ref/*.txt were produced by tests/golden/make_ref_fixtures.py running
the reference's bfp_solver (built from its sources by `make -C oracle ref-gpu`)
on a B200: sixteen small configurations covering the eq15 and legacy energy
models, straggling, lite-memory, primary-only without clipping, energy-only,
no-transport, no-angle, the golden-run beam options, the legacy cross-section
calibration, the stopping-power-only dose, bone, a non-square grid, an 8x8
square grid, and the energy-moment and spot-plane outputs.

CPU (oracle): the first steps of every case, plus the moments and a spot plane;
the full runs are opt-in (BFPN_SLOW=1).  GPU (FP64 CUDA path): every case in
full.  Tolerances: IDD 1e-12 of its peak for the oracle and 1e-10 for the GPU
path; the psi^2 proxy, a sum that cancels to ~1e-4 of its terms, 1e-9 of its
largest value; moments and spot planes 1e-5 (the reference prints 6 digits).
"""
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import GOLDEN, ROOT

sys.path.insert(0, GOLDEN)
from make_ref_fixtures import REF_CASES, TABLES  # noqa: E402

from bfpn_gpu_b200 import Context, capi, parse_args, read_tables  # noqa: E402
from oracle import oracle as O  # noqa: E402

REF = os.path.join(GOLDEN, "ref")
PREFIX = 12


def case(name):
    cfg = parse_args(REF_CASES[name].format(t=TABLES).split())
    mu, sig = read_tables(cfg.resolved_data_path(), cfg.ng)
    return cfg, mu, sig, np.loadtxt(os.path.join(REF, name + ".txt"))


def check(idd, prox, ref, idd_tol, prox_tol=1e-9):
    n = len(idd)
    scale = np.abs(ref[:, 1]).max()
    assert np.abs(idd - ref[:n, 1]).max() <= idd_tol * scale
    pscale = np.abs(ref[:, 2]).max()
    assert np.abs(prox - ref[:n, 2]).max() <= prox_tol * max(pscale, 1e-300)


@pytest.mark.parametrize("name", sorted(REF_CASES))
def test_oracle_prefix_matches_reference(name):
    cfg, mu, sig, ref = case(name)
    assert ref.shape[0] == cfg.max_steps()
    idd, prox = O.Oracle(cfg.grid(), cfg.phys(), mu, sig).step(PREFIX)
    check(idd, prox, ref, 1e-12)


@pytest.mark.slow
@pytest.mark.parametrize("name", sorted(REF_CASES))
def test_oracle_full_run_matches_reference(name):
    cfg, mu, sig, ref = case(name)
    idd, prox = O.Oracle(cfg.grid(), cfg.phys(), mu, sig).step(cfg.max_steps())
    check(idd, prox, ref, 1e-12)


def test_oracle_moments_and_spot_plane_match_reference():
    cfg, mu, sig, _ = case("moments_and_spots")
    ora = O.Oracle(cfg.grid(), cfg.phys(), mu, sig)
    mom = np.loadtxt(os.path.join(REF, "moments_and_spots_moments.txt"))
    assert mom.shape == (cfg.max_steps() * cfg.ng, 5)
    for step in range(1, 26):
        ora.step(1)
        if step <= 4:
            got = ora.energy_moments().reshape(-1, 2)
            want = mom[(step - 1) * cfg.ng: step * cfg.ng, 3:]
            assert np.abs(got - want).max() <= 1e-5 * np.abs(want).max()
    plane = np.loadtxt(os.path.join(REF, "moments_and_spots_spot_req5.00_x5.00.txt"))
    got = ora.spot_plane()
    assert plane.shape == (got.size, 3)
    assert np.abs(plane[:, 2] - got).max() <= 1e-5 * np.abs(got).max()


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(REF_CASES))
def test_gpu_fp64_full_run_matches_reference(name):
    cfg, mu, sig, ref = case(name)
    ctx = Context(cfg.grid(), cfg.phys(), capi.PREC_FP64)
    ctx.load_tables(mu, sig)
    ctx.init_beam()
    idd, prox = ctx.step(cfg.max_steps())
    check(idd, prox, ref, 1e-10)


@pytest.mark.gpu
def test_gpu_cli_moments_and_spots_match_reference(tmp_path):
    """The drop-in CLI writes the same files as the reference, to its printed digits."""
    cli = os.path.join(ROOT, "bfpn_gpu_b200", "bin", "bfp_solver")
    args = REF_CASES["moments_and_spots"].format(t=TABLES).split()
    r = subprocess.run([cli] + args, cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    ref = np.loadtxt(os.path.join(REF, "moments_and_spots.txt"))
    idd = np.loadtxt(tmp_path / "idd_output.txt")
    prox = np.loadtxt(tmp_path / "dose_output.txt")
    assert np.array_equal(idd[:, 0], ref[:, 0])
    check(idd[:, 1], prox[:, 1], ref, 1e-10)
    mom = np.loadtxt(tmp_path / "energy_moments.txt")
    want = np.loadtxt(os.path.join(REF, "moments_and_spots_moments.txt"))
    assert mom.shape == want.shape and np.array_equal(mom[:, :3], want[:, :3])
    for s in range(0, mom.shape[0], 2000):  # per step, relative to that step's largest moment
        blk = slice(s, s + 200)
        assert np.abs(mom[blk, 3:] - want[blk, 3:]).max() <= 2e-5 * np.abs(want[blk, 3:]).max()
    for fn in ("spot_req5.00_x5.00.txt", "spot_req10.10_x10.20.txt"):
        got = open(tmp_path / fn).read().splitlines()
        exp = open(os.path.join(REF, "moments_and_spots_" + fn)).read().splitlines()
        assert got[:3] == exp[:3] and len(got) == len(exp)
        g = np.loadtxt(tmp_path / fn)
        e = np.loadtxt(os.path.join(REF, "moments_and_spots_" + fn))
        assert np.array_equal(g[:, :2], e[:, :2])
        assert np.abs(g[:, 2] - e[:, 2]).max() <= 2e-5 * np.abs(e[:, 2]).max()
