"""Validation harness for the solver's depth-dose output.

Restates the reference's IDD analysis (scripts/analyze_idd.py) and its paper
Table 2 runner (scripts/run_table2.py) for this solver's CLI:

- `analyze(x, dose)`: Bragg peak BP (depth of the maximum), P90 (proximal 90 %
  crossing), D90 / D20 (distal 90 % / 20 % crossings) by linear interpolation of
  the peak-normalised curve, and Dmax (analyze_idd.py:21-62);
- `entrance(x, dose)`: the peak-normalised dose of the first depth (the
  "norm0" column of results/stage6_final_water230/summary.md);
- `run_table2(...)`: the six water / bone x 50 / 100 / 230 MeV cases through
  bfp_solver, each analysed and compared with Table 2.

    python -m bfpn_gpu_b200.validation analyze -i idd_output.txt --material water --energy 230
    python -m bfpn_gpu_b200.validation table2 --nx 1000 --outdir table2_runs
"""
import argparse
import math
import os
import shutil
import subprocess
import sys

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
CLI = os.path.join(_PKG, "bin", "bfp_solver")

# Paper Table 2 positions in cm (scripts/analyze_idd.py:11-18).
TABLE2 = {
    ("water", 50): {"BP": 2.150, "P90": 2.075, "D90": 2.205, "D20": 2.345},
    ("water", 100): {"BP": 7.560, "P90": 7.418, "D90": 7.671, "D20": 7.945},
    ("water", 230): {"BP": 32.540, "P90": 32.172, "D90": 32.828, "D20": 33.513},
    ("bone", 50): {"BP": 1.360, "P90": 1.319, "D90": 1.402, "D20": 1.488},
    ("bone", 100): {"BP": 4.770, "P90": 4.675, "D90": 4.837, "D20": 5.005},
    ("bone", 230): {"BP": 20.390, "P90": 20.168, "D90": 20.585, "D20": 21.023},
}
TABLE2_CASES = [("water", 50), ("water", 100), ("water", 230), ("bone", 50), ("bone", 100), ("bone", 230)]


def _cross(x0, y0, x1, y1, target):
    if y1 == y0:
        return x0
    return x0 + (target - y0) / (y1 - y0) * (x1 - x0)


def _left_crossing(x, y, peak, target):
    """First rising crossing of `target` walking left from the peak."""
    for i in range(peak, 0, -1):
        y0, y1 = y[i - 1], y[i]
        if (y0 - target) * (y1 - target) <= 0 and y0 <= target <= y1:
            return _cross(x[i - 1], y0, x[i], y1, target)
    return math.nan


def _right_crossing(x, y, peak, target):
    """First falling crossing of `target` walking right from the peak."""
    for i in range(peak, len(x) - 1):
        y0, y1 = y[i], y[i + 1]
        if (y0 - target) * (y1 - target) <= 0 and y0 >= target >= y1:
            return _cross(x[i], y0, x[i + 1], y1, target)
    return math.nan


def analyze(x, dose):
    """{"BP", "P90", "D90", "D20", "Dmax"} of one IDD curve (finite samples only)."""
    x = np.asarray(x, dtype=np.float64)
    dose = np.asarray(dose, dtype=np.float64)
    keep = np.isfinite(x) & np.isfinite(dose)
    x, dose = x[keep], dose[keep]
    if x.size == 0:
        raise ValueError("no finite IDD samples")
    if np.max(dose) <= 0:
        raise ValueError("IDD has no positive dose values")
    peak = int(np.argmax(dose))
    dmax = float(dose[peak])
    norm = dose / dmax
    return {"BP": float(x[peak]), "P90": _left_crossing(x, norm, peak, 0.9),
            "D90": _right_crossing(x, norm, peak, 0.9), "D20": _right_crossing(x, norm, peak, 0.2), "Dmax": dmax}


def entrance(x, dose):
    """Peak-normalised dose at the first depth sample."""
    dose = np.asarray(dose, dtype=np.float64)
    return float(dose[0] / np.max(dose))


def peak_depth(idd, dx):
    """Depth (cm) of the IDD maximum of a run whose row i lies at (i+1)*dx,
    refined by the parabola through the maximum sample and its two
    neighbours (sub-step resolution)."""
    idd = np.asarray(idd, dtype=np.float64)
    i = int(np.argmax(idd))
    x = (i + 1) * dx
    if 0 < i < len(idd) - 1:
        y0, y1, y2 = idd[i - 1], idd[i], idd[i + 1]
        den = y0 - 2 * y1 + y2
        if den != 0:
            x += 0.5 * dx * (y0 - y2) / den
    return x


# Accuracy bar of a reduced-precision run against an FP64 run of the same
# beam: the IDD within 0.1 % at every depth where the FP64 dose exceeds 1 % of
# its peak, and the Bragg peak within 0.1 mm.
IDD_REL_TOL = 1e-3
PEAK_FLOOR = 0.01
BRAGG_SHIFT_TOL_MM = 0.1


def idd_accuracy(idd, idd_fp64, dx):
    """IDD error of `idd` against the FP64 curve of the same beam (same
    depth grid of step dx cm): the worst pointwise relative error above
    PEAK_FLOOR of the peak, the worst error relative to the peak, the
    Bragg-peak shift in mm, and whether the bar above is met."""
    a = np.asarray(idd, dtype=np.float64)
    b = np.asarray(idd_fp64, dtype=np.float64)
    if a.shape != b.shape or a.size == 0:
        raise ValueError("IDD curves differ in length or are empty")
    peak = float(np.abs(b).max())
    big = b > PEAK_FLOOR * peak
    rel = float((np.abs(a - b)[big] / b[big]).max())
    shift = abs(peak_depth(a, dx) - peak_depth(b, dx)) * 10.0
    return {"steps": int(b.size), "idd_max_rel_err_above_1pct_peak": rel,
            "idd_max_err_rel_to_peak": float(np.abs(a - b).max() / peak),
            "bragg_peak_cm_fp64": float(peak_depth(b, dx)), "bragg_peak_shift_mm": float(shift),
            "criterion": "rel err <= %g above %g of peak, Bragg-peak shift <= %g mm"
                         % (IDD_REL_TOL, PEAK_FLOOR, BRAGG_SHIFT_TOL_MM),
            "pass": bool(rel <= IDD_REL_TOL and shift <= BRAGG_SHIFT_TOL_MM)}


def load_idd(path):
    data = np.loadtxt(path, comments="#", ndmin=2)
    if data.shape[1] < 2:
        raise ValueError("%s must have at least two columns: x dose" % path)
    return data[:, 0], data[:, 1]


def format_table(metrics, reference=None):
    lines = ["metric   gpu_cm      paper_cm    diff_cm     rel_diff_pct"]
    for name in ("BP", "P90", "D90", "D20"):
        v = metrics[name]
        ref = reference.get(name) if reference else None
        if ref is None or math.isnan(v):
            lines.append("%-6s %10.4f %10s %10s %14s" % (name, v, "-", "-", "-"))
        else:
            lines.append("%-6s %10.4f %10.4f %10.4f %14.4f" % (name, v, ref, v - ref, (v - ref) / ref * 100.0))
    lines.append("Dmax   %10.6g" % metrics["Dmax"])
    return "\n".join(lines)


def run_table2(exe=CLI, nx=4000, time=40.0, outdir="table2_runs", paper_grid=False, skip_run=False,
               extra_args=(), cwd=None):
    """Run (unless skip_run) and analyse the six Table 2 cases; returns
    {(material, energy): metrics} and writes <outdir>/summary.txt."""
    cwd = cwd or os.getcwd()
    outdir = os.path.join(cwd, outdir)
    os.makedirs(outdir, exist_ok=True)
    results = {}
    with open(os.path.join(outdir, "summary.txt"), "w") as summary:
        for material, energy in TABLE2_CASES:
            case = os.path.join(outdir, "%s_%d" % (material, energy))
            os.makedirs(case, exist_ok=True)
            idd_path = os.path.join(case, "idd_output.txt")
            if not skip_run:
                cmd = [exe, str(nx), "--time", str(time), "--material", material, "--energy", str(energy)]
                if paper_grid:
                    cmd += ["--ny", "80", "--nz", "80", "--nmu", "20", "--nom", "20"]
                cmd += list(extra_args)
                print("+", " ".join(cmd), flush=True)
                subprocess.run(cmd, cwd=case, check=True)
            x, dose = load_idd(idd_path)
            m = analyze(x, dose)
            results[(material, energy)] = m
            block = "\n[%s %d MeV]\n%s\n" % (material, energy, format_table(m, TABLE2[(material, energy)]))
            print(block)
            summary.write(block)
    return results


def main(argv=None):
    ap = argparse.ArgumentParser(description="IDD validation: BP/P90/D90/D20 metrics and the Table 2 runner")
    sub = ap.add_subparsers(dest="cmd", required=True)
    a = sub.add_parser("analyze", help="metrics of one idd_output.txt")
    a.add_argument("-i", "--input", default="idd_output.txt")
    a.add_argument("--material", choices=["water", "bone"])
    a.add_argument("--energy", type=int, choices=[50, 100, 230])
    t = sub.add_parser("table2", help="run and analyse the six Table 2 cases")
    t.add_argument("--exe", default=CLI)
    t.add_argument("--nx", type=int, default=4000)
    t.add_argument("--time", type=float, default=40.0)
    t.add_argument("--outdir", default="table2_runs")
    t.add_argument("--paper-grid", action="store_true", help="80x80 space and 20x20 angle grid")
    t.add_argument("--skip-run", action="store_true", help="only analyse existing outputs")
    t.add_argument("--precision", choices=["fp64", "mixed"], default=None)
    args = ap.parse_args(argv)
    if args.cmd == "analyze":
        if bool(args.material) != bool(args.energy):
            print("--material and --energy must be provided together for Table 2 comparison", file=sys.stderr)
            return 2
        x, dose = load_idd(args.input)
        ref = TABLE2[(args.material, args.energy)] if args.material else None
        print(format_table(analyze(x, dose), ref))
        return 0
    extra = ["--precision", args.precision] if args.precision else []
    run_table2(args.exe, args.nx, args.time, args.outdir, args.paper_grid, args.skip_run, extra)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
