"""The IDD validation harness (bfpn_gpu_b200.validation) against the numbers the
reference published for its own golden runs
(results/stage6_final_water230/summary.md:11-14: norm0, BP, P90, D90, D20 to the
printed digits), and its Table 2 runner on a stand-in solver."""
import os
import stat
import sys

import numpy as np
import pytest

from conftest import load_golden
from bfpn_gpu_b200 import validation as V

SUMMARY = {  # grid: (norm0, BP, P90, D90, D20)
    "8_7": (0.218797169, 32.5600, 32.3066, 32.7443, 33.2153),
    "12_9": (0.218866538, 32.5600, 32.3051, 32.7437, 33.2150),
}


@pytest.mark.parametrize("grid", ["8_7", "12_9"])
def test_metrics_of_the_golden_runs(grid):
    d = load_golden(grid)
    m = V.analyze(d[:, 0], d[:, 1])
    norm0, bp, p90, d90, d20 = SUMMARY[grid]
    assert round(V.entrance(d[:, 0], d[:, 1]), 9) == norm0
    for k, v in (("BP", bp), ("P90", p90), ("D90", d90), ("D20", d20)):
        assert round(m[k], 4) == v, (k, m[k], v)


def test_crossings_on_an_analytic_curve():
    x = np.linspace(0.0, 10.0, 1001)
    dose = np.exp(-0.5 * ((x - 6.0) / 0.5) ** 2)
    m = V.analyze(x, dose)
    half = 0.5 * np.sqrt(-2 * np.log(0.9))
    assert m["BP"] == pytest.approx(6.0)
    assert m["P90"] == pytest.approx(6.0 - half, abs=1e-4)
    assert m["D90"] == pytest.approx(6.0 + half, abs=1e-4)
    assert m["D20"] == pytest.approx(6.0 + 0.5 * np.sqrt(-2 * np.log(0.2)), abs=1e-4)
    with pytest.raises(ValueError):
        V.analyze(x, -dose)


def test_cli_table_against_paper(tmp_path, capsys):
    d = load_golden("8_7")
    path = tmp_path / "idd.txt"
    np.savetxt(path, d[:, :2], header="x_cm value")
    assert V.main(["analyze", "-i", str(path), "--material", "water", "--energy", "230"]) == 0
    out = capsys.readouterr().out
    assert "BP" in out and "32.5400" in out and "Dmax" in out
    assert V.main(["analyze", "-i", str(path), "--material", "water"]) == 2


def test_table2_runner_with_a_stand_in_solver(tmp_path):
    """run_table2 drives the solver once per case (reference CLI arguments) and
    analyses what it wrote."""
    fake = tmp_path / "fake_solver.py"
    fake.write_text(
        "import sys, numpy as np\n"
        "a = sys.argv[1:]\n"
        "e = float(a[a.index('--energy') + 1]); rho = 1.0 if a[a.index('--material') + 1] == 'water' else 1.85\n"
        "x = np.arange(1, 4001) * 0.01\n"
        "r = 0.0022 * e ** 1.77 / rho\n"
        "d = 1 + np.exp(-0.5 * ((x - r) / 0.1) ** 2) * 4\n"
        "d[x > r + 0.5] = 0\n"
        "np.savetxt('idd_output.txt', np.c_[x, d], header='x_cm value')\n")
    exe = tmp_path / "solver"
    exe.write_text("#!/bin/sh\nexec %s %s \"$@\"\n" % (sys.executable, fake))
    exe.chmod(exe.stat().st_mode | stat.S_IEXEC)
    res = V.run_table2(exe=str(exe), nx=4000, time=40.0, outdir="t2", cwd=str(tmp_path))
    assert set(res) == set(V.TABLE2_CASES)
    for (mat, e), m in res.items():
        assert m["BP"] == pytest.approx(0.0022 * e ** 1.77 / (1.0 if mat == "water" else 1.85), abs=0.011)
    assert os.path.exists(tmp_path / "t2" / "summary.txt")
    # analysis only, on the outputs just written
    again = V.run_table2(exe="/nonexistent", outdir="t2", cwd=str(tmp_path), skip_run=True)
    assert again == res


def test_accuracy_metric_flags_a_planted_error():
    """The criterion itself, on the CPU: a 0.2 % bump above 1 % of the peak
    or a one-step peak shift fails; a bump in the tail below 1 % passes."""
    x = np.arange(1, 1001) * 0.04
    ref = np.exp(-0.5 * ((x - 30.0) / 1.5) ** 2) + 0.2 * (x < 30.0)
    ok = ref * (1 + 5e-4)
    assert V.idd_accuracy(ok, ref, 0.04)["pass"]
    bad = ref.copy()
    bad[500] *= 1.002
    assert not V.idd_accuracy(bad, ref, 0.04)["pass"]
    tail = ref.copy()
    tail[-1] *= 1.5  # the tail is below 1 % of the peak
    assert ref[-1] < 0.01 * ref.max() and V.idd_accuracy(tail, ref, 0.04)["pass"]
    shifted = np.roll(ref, 1)
    assert V.idd_accuracy(shifted, ref, 0.04)["bragg_peak_shift_mm"] > V.BRAGG_SHIFT_TOL_MM
