"""Golden fixtures from the reference's own CUDA solver.

Runs oracle/_ref/bfp_solver_ref (built from the reference's sources by
`make -C oracle ref-gpu`) on a GPU host for the small configurations in
REF_CASES and writes, per case, <out>/<name>.txt with columns
x_cm, IDD, dose proxy (17 significant digits, as the solver printed them), plus
<name>_moments.txt / <name>_spot_*.txt where the case asks for them.  The
fixtures are committed under tests/golden/ref/; tests compare the oracle (CPU)
and the CUDA path against them.

    python tests/golden/make_ref_fixtures.py --out <dir>
"""
import argparse
import os
import shutil
import subprocess
import sys
import tempfile

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
BIN = os.path.join(ROOT, "oracle", "_ref", "bfp_solver_ref")
TABLES = os.path.join(ROOT, "tests", "golden", "tables")

# 100 depth steps of 0.2 cm, 150 MeV protons, small transverse / angular grids.
BASE = ("200 --time 20 --energy 150 --sigma-e 1.5 --sigma-yz 0.4 --ny 6 --nz 6 --ly 4 --lz 4 "
        "--nmu 5 --nom 5 --ng 200")
WATER = "--data {t}/water --material water"
REF_CASES = {
    "eq15": BASE + " " + WATER,
    "eq15_straggling": BASE + " " + WATER + " --eq15-straggling",
    "legacy_energy": BASE + " " + WATER + " --energy-model legacy",
    "legacy_energy_straggling": BASE + " " + WATER + " --energy-model legacy --eq15-straggling",
    "lite_memory": BASE + " " + WATER + " --lite-memory",
    "primary_only_no_clipping": BASE + " " + WATER + " --primary-only --no-spatial-clipping",
    "energy_only": BASE + " " + WATER + " --energy-only",
    "no_transport": BASE + " " + WATER + " --no-transport",
    "no_angle": BASE + " " + WATER + " --no-angle",
    "trapezoidal_delta_normalized": BASE + " " + WATER +
    " --trapezoidal-yz --discrete-angle-delta --normalize-initial-mass",
    "legacy_cross_section": BASE + " " + WATER + " --legacy-cross-section-calibration",
    "stopping_power_dose_only": BASE + " " + WATER + " --stopping-power-dose-only",
    "bone": BASE + " --data {t}/bone --material bone --rho 1.85",
    "odd_grid": ("150 --time 15 --energy 120 --sigma-e 1.2 --sigma-yz 0.3 --ny 7 --nz 5 --ly 3 --lz 2.5 "
                 "--nmu 4 --nom 6 --ng 150 " + WATER),
    "square_8x8": ("120 --time 12 --energy 100 --sigma-e 1.0 --sigma-yz 0.5 --ny 8 --nz 8 --ly 4 --lz 4 "
                   "--nmu 8 --nom 8 --ng 120 " + WATER),
    "moments_and_spots": BASE + " " + WATER + " --save-energy-moments --spot-depths 5,10.1 --spot-prefix spot",
}


def run_case(name, args, out):
    argv = [BIN] + args.format(t=TABLES).split()
    with tempfile.TemporaryDirectory() as d:
        r = subprocess.run(argv, cwd=d, capture_output=True, text=True, timeout=600)
        if r.returncode != 0:
            raise RuntimeError("%s failed (%d): %s" % (name, r.returncode, (r.stderr or r.stdout)[-2000:]))
        idd = open(os.path.join(d, "idd_output.txt")).read().splitlines()
        prox = open(os.path.join(d, "dose_output.txt")).read().splitlines()
        assert idd[0].startswith("#") and len(idd) == len(prox)
        with open(os.path.join(out, name + ".txt"), "w") as f:
            f.write("# reference bfp_solver %s\n# x_cm idd proxy\n" % args.replace("{t}", "<tables>"))
            for a, b in zip(idd[1:], prox[1:]):
                x, v = a.split()
                f.write("%s %s %s\n" % (x, v, b.split()[1]))
        if os.path.exists(os.path.join(d, "energy_moments.txt")):
            shutil.copy(os.path.join(d, "energy_moments.txt"), os.path.join(out, name + "_moments.txt"))
        for fn in sorted(os.listdir(d)):
            if fn.startswith("spot_"):
                shutil.copy(os.path.join(d, fn), os.path.join(out, name + "_" + fn))
    return len(idd) - 1


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--only", default=None, help="comma-separated case names")
    a = ap.parse_args()
    if not os.path.exists(BIN):
        sys.exit("%s is missing: build it with make -C oracle ref-gpu" % BIN)
    os.makedirs(a.out, exist_ok=True)
    names = a.only.split(",") if a.only else list(REF_CASES)
    for n in names:
        print(n, run_case(n, REF_CASES[n], a.out), "steps", flush=True)


if __name__ == "__main__":
    main()
