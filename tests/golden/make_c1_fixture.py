"""Writes tests/golden/idd_c1_oracle.txt: the oracle's FP64 IDD and dose proxy
for the 100 MeV configuration (water, sigma_E 1 MeV, sigma_yz 0.4 cm, 4 x 4 cm,
Ny = Nz = 16, Nmu = Nom = 8, Ng = 200 over Lg = 104 MeV with the reference's
synthetic tables generated for -n 200 -l 104, 10 cm depth at Nx = 1000, eq15
with secondaries).  The oracle itself is pinned by test_oracle_golden.py.

Usage: python tests/golden/make_c1_fixture.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

C1_ARGS = ("1000 --time 10 --material water --energy 100 --sigma-e 1.0 --sigma-yz 0.4 --ly 4 --lz 4 "
           "--ny 16 --nz 16 --nmu 8 --nom 8 --ng 200 --lg 104")


def main():
    from bfpn_gpu_b200 import parse_args, read_tables
    from oracle import oracle as O
    cfg = parse_args(C1_ARGS.split())
    mu, sig = read_tables(os.path.join(HERE, "tables", "synthetic200_lg104"), cfg.ng)
    o = O.Oracle(cfg.grid(), cfg.phys(), mu, sig)
    idd, proxy = o.step(cfg.max_steps())
    x = (np.arange(len(idd)) + 1) * cfg.dt()
    np.savetxt(os.path.join(HERE, "idd_c1_oracle.txt"), np.c_[x, idd, proxy], fmt="%.17g",
               header="oracle FP64: " + C1_ARGS + "\nx_cm idd proxy")


if __name__ == "__main__":
    main()
