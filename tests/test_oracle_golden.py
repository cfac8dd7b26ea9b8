"""The oracle against the reference's own golden IDD output.

results/stage6_final_water230/{8_7,12_9}_nx1000/idd_output.txt were written by
the reference's eq15 path (17 significant digits).  The CPU restatement must
reproduce them to rounding: a relative difference below 1e-12 per row.
"""
import numpy as np
import pytest

from conftest import golden_config, load_golden, material_tables
from oracle import oracle as O


@pytest.mark.parametrize("grid,steps", [("8_7", 6), ("12_9", 3)])
def test_oracle_matches_reference_golden_prefix(grid, steps):
    cfg = golden_config(grid)
    mu, sig = material_tables(cfg, "water")
    o = O.Oracle(cfg.grid(), cfg.phys(), mu, sig)
    idd, _ = o.step(steps)
    gold = load_golden(grid)
    np.testing.assert_allclose(gold[:steps, 0], (np.arange(steps) + 1) * cfg.dt(), rtol=0, atol=1e-15)
    rel = np.abs(idd - gold[:steps, 1]) / np.abs(gold[:steps, 1])
    assert rel.max() < 1e-12, rel


@pytest.mark.slow
@pytest.mark.parametrize("grid", ["8_7", "12_9"])
def test_oracle_matches_reference_golden_full(grid):
    cfg = golden_config(grid)
    mu, sig = material_tables(cfg, "water")
    o = O.Oracle(cfg.grid(), cfg.phys(), mu, sig)
    idd, _ = o.step(cfg.max_steps())
    gold = load_golden(grid)
    assert np.abs(idd - gold[:, 1]).max() / np.abs(gold[:, 1]).max() < 1e-11


def test_c1_fixture_matches_current_oracle_prefix():
    """tests/golden/idd_c1_oracle.txt (full 250-step oracle run, made by
    tests/golden/make_c1_fixture.py) agrees with the oracle as built."""
    import os
    from conftest import GOLDEN, table_dir
    from bfpn_gpu_b200 import parse_args, read_tables
    fx = os.path.join(GOLDEN, "idd_c1_oracle.txt")
    args = open(fx).readline().split("oracle FP64:")[1].split()
    cfg = parse_args(args)
    ref = np.loadtxt(fx)
    mu, sig = read_tables(table_dir("synthetic200_lg104"), cfg.ng)
    o = O.Oracle(cfg.grid(), cfg.phys(), mu, sig)
    idd, proxy = o.step(3)
    assert np.array_equal(idd, ref[:3, 1]) and np.array_equal(proxy, ref[:3, 2])


def test_oracle_lite_memory_mode_runs():
    """Lite-memory restatement: psi^1 only, attenuating, proxy 0."""
    from bfpn_gpu_b200 import make_config
    cfg = make_config(nx=100, ny=4, nz=4, nmu=3, nom=3, ng=40, lg=59.0, beam_energy=40.0, sigma_e=2.0,
                      sigma_yz=0.4, ly=2.0, lz=2.0, lite_memory=True, t_final=2.0)
    mu, sig = material_tables(cfg, "synthetic500")
    ora = O.Oracle(cfg.grid(), cfg.phys(), mu, sig)
    m0 = ora.get_state(0, 0).sum()
    idd, prox = ora.step(10)
    assert np.all(idd > 0) and not np.any(prox)
    assert 0 < ora.get_state(0, 0).sum() < m0
    assert not np.any(ora.get_state(0, 1)) and not np.any(ora.get_state(1, 0))
