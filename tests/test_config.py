"""Command-line semantics of the reference's main (src/main.cu:44-356), both
in the Python parser and in the native CLI (--print-config, no GPU used)."""
import json
import os
import subprocess

import pytest

from conftest import ROOT
from bfpn_gpu_b200 import capi, parse_args
from bfpn_gpu_b200.config import ArgError

CLI = os.path.join(ROOT, "bfpn_gpu_b200", "bin", "bfp_solver")


def test_defaults_match_reference():
    c = parse_args([])
    assert (c.nx, c.ny, c.nz, c.ng, c.nmu, c.nom) == (4000, 10, 10, 500, 11, 11)
    assert (c.ly, c.lz, c.lu, c.lv, c.lg) == (1.0, 1.0, 1.0, 1.0, 259.0)
    assert c.t_final == 40.0 and c.beam_energy == 230.0 and c.sigma_e == 1.0 and c.sigma_yz == 0.1
    assert c.dose_catastrophic_loss and not c.calibrate_cross_sections and not c.legacy_energy
    assert c.resolved_data_path() == "./data"


def test_material_resets_rho_and_sets_data_path():
    c = parse_args("--rho 1.85 --material bone".split())
    assert c.density == 1.757 and c.energy_density == 1.757
    c = parse_args("--material bone --rho 1.85".split())
    assert c.density == 1.85 and c.energy_density == 1.85
    assert c.resolved_data_path() == "BFPn_CPU_Solver/bone"
    c = parse_args("--material air --data /x".split())
    assert c.resolved_data_path() == "/x" and c.density == 0.001205
    with pytest.raises(ArgError):
        parse_args("--material lead".split())


def test_positional_nx_and_steps():
    c = parse_args("1000 --time 10".split())
    assert c.nx == 1000 and abs(c.dt() - 0.04) < 1e-15 and c.max_steps() == 250
    assert parse_args("2000 --time 8.0".split()).max_steps() == 400


def test_flags():
    c = parse_args("--energy-model legacy --stopping-power-dose-only --legacy-cross-section-calibration "
                   "--primary-only --no-angle --trapezoidal-yz".split())
    f = c.flags()
    assert f & capi.FLAG_LEGACY_ENERGY and f & capi.FLAG_PRIMARY_ONLY and f & capi.FLAG_NO_ANGLE
    assert f & capi.FLAG_CALIBRATE_CROSS_SECTIONS and f & capi.FLAG_TRAPEZOIDAL_YZ
    assert not f & capi.FLAG_DOSE_CATASTROPHIC_LOSS
    with pytest.raises(ArgError):
        parse_args("--energy-model foo".split())
    with pytest.raises(ArgError):
        parse_args("--lite-memory --streaming-full".split())
    p = parse_args("--sigma-yz 0.3".split()).phys()
    assert p.a_1 == 1.0 / 2.0 / 0.3 / 0.3 and p.a_2 == 1.0 / 2.0 / 1e-6 / 1e-6


CASES = [
    "",
    "1000 --time 40 --material water --energy 230 --ny 8 --nz 8 --nmu 7 --nom 7 --ly 8 --lz 8 --lu 2 --lv 2 "
    "--sigma-yz 0.3 --discrete-angle-delta --normalize-initial-mass --trapezoidal-yz",
    "--material bone --rho 1.85 --ny 80 --nz 80 --nmu 20 --nom 20 --ly 16 --lz 16 --precision mixed",
    "1000 --time 10 --data tests/golden/tables/synthetic200_lg104 --lg 104 --ng 200 --energy 100 --sigma-e 1.0 "
    "--ny 16 --nz 16 --nmu 8 --nom 8 --ly 4 --lz 4 --sigma-yz 0.4",
    "--energy-model legacy --eq15-straggling --no-transport --no-spatial-clipping --stopping-power-dose-only",
    "--rho 2.0 --material air --energy-only --primary-only --no-angle --legacy-cross-section-calibration",
]


@pytest.mark.parametrize("argv", CASES)
def test_native_cli_parses_like_python(argv):
    args = argv.split()
    out = subprocess.run([CLI] + args + ["--print-config"], check=True, capture_output=True, text=True).stdout
    js = json.loads(out)
    c = parse_args(args)
    g, p = c.grid(), c.phys()
    assert js["data_path"] == c.resolved_data_path()
    assert js["t_final"] == c.t_final
    for k in ("Nx", "Ny", "Nz", "Ng", "Nmu", "Nom", "Lx", "Ly", "Lz", "Lu", "Lv", "Lg"):
        assert js[k] == getattr(g, k), k
    for k in ("sig_E", "a_1", "a_2", "beam_energy", "density", "energy_density", "material", "flags"):
        assert js[k] == getattr(p, k), k
    assert js["precision"] == c.precision


def test_native_cli_help_and_errors():
    r = subprocess.run([CLI, "--help"], capture_output=True, text=True)
    assert r.returncode == 0 and "--energy-model" in r.stdout
    r = subprocess.run([CLI, "--material", "lead"], capture_output=True, text=True)
    assert r.returncode == 1 and "Unknown material: lead" in r.stderr
    r = subprocess.run([CLI, "--lite-memory", "--streaming-full"], capture_output=True, text=True)
    assert r.returncode == 1
