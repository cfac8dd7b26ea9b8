"""Regenerates the committed fixtures under tests/golden/ from the reference
tree (xiaojin1423764/BFPn_GPU), which must be present at REF_ROOT.

* idd_water230_{8_7,12_9}_nx1000.txt -- the reference's own 17-digit IDD output
  (results/stage6_final_water230/*/idd_output.txt), the pins of the oracle.
* tables/{water,bone,air,synthetic500}/ -- the material tables the reference
  reads (BFPn_CPU_Solver/<material>/, data/), copied byte for byte.
* tables/synthetic200_lg104/ -- scripts/generate_test_data.py run with
  -n 200 -l 104 (imported from the reference tree, executed here), the inputs
  of the 100 MeV FP64 configuration.

Usage: python tests/golden/make_fixtures.py [REF_ROOT]
"""
import importlib.util
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref_root):
    res = os.path.join(ref_root, "results", "stage6_final_water230")
    for grid in ("8_7", "12_9"):
        shutil.copyfile(os.path.join(res, grid + "_nx1000", "idd_output.txt"),
                        os.path.join(HERE, "idd_water230_%s_nx1000.txt" % grid))
    copies = {
        "water": ("BFPn_CPU_Solver/water", ["data_cross.txt", "cross_total.txt"]),
        "bone": ("BFPn_CPU_Solver/bone", ["data_b.txt", "cross_total.txt"]),
        "air": ("BFPn_CPU_Solver/air", ["data_a.txt", "cross_total.txt"]),
        "synthetic500": ("data", ["data_cross.txt", "cross_total.txt"]),
    }
    for name, (sub, files) in copies.items():
        dst = os.path.join(HERE, "tables", name)
        os.makedirs(dst, exist_ok=True)
        for f in files:
            shutil.copyfile(os.path.join(ref_root, sub, f), os.path.join(dst, f))
    spec = importlib.util.spec_from_file_location("ref_gen", os.path.join(ref_root, "scripts", "generate_test_data.py"))
    gen = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(gen)
    dst = os.path.join(HERE, "tables", "synthetic200_lg104")
    os.makedirs(dst, exist_ok=True)
    gen.generate_cross_sections(200, 104.0, dst)
    for f in os.listdir(dst):  # the generator may also write a plot when matplotlib exists
        if not f.endswith(".txt"):
            os.remove(os.path.join(dst, f))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
