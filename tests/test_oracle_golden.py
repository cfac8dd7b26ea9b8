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
