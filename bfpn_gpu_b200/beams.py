"""Beam request sets for batching and serving.

`uneven_beams` draws independent pencil beams from a seed: energy uniform in
70-230 MeV, water or bone with probability 1/2 each, transverse sigma uniform in
0.3-0.8 cm, Ny = Nz from {16, 32, 48, 64}, Nmu = Nom from {12, 16, 20}, about 2
energy groups per MeV over E0 + 10 MeV, and a depth of 1.2 times the CSDA range
computed from the same stopping-power table the solver builds (depth step
0.04 cm).  `poisson_arrivals` gives request times for a serving run.
"""
import math
import os

import numpy as np

from . import capi
from .config import make_config

_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TABLE_ROOT = os.path.join(_ROOT, "tests", "golden", "tables")
DENSITY = {"water": 1.0, "bone": 1.85}


def csda_range_cm(cfg, mu, sigma):
    """Continuous-slowing-down range of the beam energy in cm: the integral of
    dE / S(E) over the DG nodes below E0, over the density."""
    # the stopping-power table does not depend on the transverse / angular grid:
    # build it on a 1-direction grid (the angular kernel is then trivial)
    g = cfg.grid()
    g.Ny = g.Nz = 1
    g.Nmu = g.Nom = 1
    S = capi.host_table(g, cfg.phys(), mu, sigma, capi.TABLE_S_S)
    en = capi.host_table(g, cfg.phys(), mu, sigma, capi.TABLE_EN)
    keep = en[1:] <= cfg.beam_energy
    r = np.sum((en[1:] - en[:-1])[keep] / (0.5 * (S[1:] + S[:-1]))[keep])
    return float(r / cfg.density)


class BeamRequest:
    """One beam: its run configuration, tables and depth-step count."""

    def __init__(self, cfg, mu, sigma, nsteps, precision):
        self.cfg, self.mu, self.sigma, self.nsteps, self.precision = cfg, mu, sigma, nsteps, precision

    @property
    def cells(self):
        c = self.cfg
        return (c.ny + 1) * (c.nz + 1) * c.nmu * c.nom * c.ng

    def beam(self):
        return capi.make_beam(self.cfg.grid(), self.cfg.phys(), self.mu, self.sigma, self.nsteps, self.precision)


def uneven_beams(n=64, seed=20261203, ny_choices=(16, 32, 48, 64), na_choices=(12, 16, 20),
                 precision=capi.PREC_MIXED, dt=0.04, table_root=TABLE_ROOT):
    rng = np.random.default_rng(seed)
    tables = {}
    out = []
    for _ in range(n):
        energy = float(rng.uniform(70.0, 230.0))
        material = "water" if rng.random() < 0.5 else "bone"
        sigma_yz = float(rng.uniform(0.3, 0.8))
        ny = int(rng.choice(ny_choices))
        na = int(rng.choice(na_choices))
        ng = int(round(2.0 * energy))
        rho = DENSITY[material]
        nx = int(round(40.0 / dt))
        cfg = make_config(nx=nx, t_final=40.0, ny=ny, nz=ny, nmu=na, nom=na, ng=ng, lg=energy + 10.0,
                          ly=8.0, lz=8.0, beam_energy=energy, sigma_e=0.01 * energy, sigma_yz=sigma_yz,
                          material_name=material, density=rho, energy_density=rho)
        key = (material, ng)
        if key not in tables:
            tables[key] = capi.read_tables(os.path.join(table_root, material), ng)
        mu, sig = tables[key]
        depth = 1.2 * csda_range_cm(cfg, mu, sig)
        cfg.t_final = depth
        out.append(BeamRequest(cfg, mu, sig, int(math.ceil(depth / cfg.dt() - 1e-12)), precision))
    return out


def poisson_arrivals(n, rate, seed=20261203):
    """n arrival times (seconds from 0) of a Poisson stream of the given rate."""
    rng = np.random.default_rng(seed + 1)
    return np.cumsum(rng.exponential(1.0 / rate, size=n))
