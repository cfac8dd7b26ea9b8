import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
TABLES = os.path.join(GOLDEN, "tables")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")
    config.addinivalue_line("markers", "slow: long CPU oracle runs; opt in with BFPN_SLOW=1")


def pytest_collection_modifyitems(config, items):
    if os.environ.get("BFPN_SLOW") == "1":
        return
    skip = pytest.mark.skip(reason="slow oracle run; set BFPN_SLOW=1")
    for it in items:
        if "slow" in it.keywords:
            it.add_marker(skip)


def table_dir(name):
    return os.path.join(TABLES, name)


# Flags of the reference's golden water 230 MeV runs
# (results/stage6_final_water230/summary.md:5-9).
GOLDEN_ARGS = ("1000 --time 40 --material water --energy 230 --ly 8 --lz 8 --lu 2 --lv 2 --sigma-yz 0.3 "
               "--discrete-angle-delta --normalize-initial-mass --trapezoidal-yz")


def golden_config(grid):
    from bfpn_gpu_b200 import parse_args
    ny, nmu = {"8_7": (8, 7), "12_9": (12, 9)}[grid]
    return parse_args((GOLDEN_ARGS + " --ny %d --nz %d --nmu %d --nom %d" % (ny, ny, nmu, nmu)).split())


def load_golden(grid):
    return np.loadtxt(os.path.join(GOLDEN, "idd_water230_%s_nx1000.txt" % grid))


def material_tables(cfg, name="water"):
    from bfpn_gpu_b200 import read_tables
    return read_tables(table_dir(name), cfg.ng)


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    scale = max(np.abs(b).max(), 1e-300)
    return float(np.abs(a - b).max() / scale)
