"""Extract the coax impedance-test fixture of the reference into a small golden file.

Source: the reference's calibration run test/校正/result_deg0.csv and result_deg5.csv
(written by OutputModule::output_phase, outputModule.hpp:38-184, after
solve_Microwave_impedanceTest, emfieldModule.hpp:5528-6099, on the grid of
test/校正/setup.yaml: ni=194, nj=7, x in [0, 0.0388], r in [0.0006, 0.002],
fmw=4.25e9, Pmw=8, Z0=50, J1r_exc=0.212687, epsr_diele=2.083825280349).
Columns kept: i, j, x, r, Er(R), Er(I), Er_anly(R), Er_anly(I) of phase snapshots 0 and 5.
Usage: python <this script> <reference checkout>  (or set CATHODE_REFERENCE).
"""
import csv
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def reference_root() -> str:
    """The reference checkout: the first command-line argument, else $CATHODE_REFERENCE."""
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("CATHODE_REFERENCE")
    if not root or not os.path.isdir(root):
        sys.exit(f"usage: python {os.path.basename(__file__)} <reference checkout> (or set CATHODE_REFERENCE)")
    return root
KEEP = ["i", "j", "x", "r", "Er(R)", "Er(I)", "Er_anly(R)", "Er_anly(I)"]


def main():
    SRC = os.path.join(reference_root(), "test", "校正")
    for n in (0, 5):
        rows = list(csv.DictReader(open(os.path.join(SRC, f"result_deg{n}.csv"))))
        out = os.path.join(HERE, f"coax_er_deg{n}.csv")
        with open(out, "w", newline="") as f:
            w = csv.writer(f)
            w.writerow(KEEP)
            for r in rows:
                w.writerow([r[k] for k in KEEP])
        print(out, len(rows))


if __name__ == "__main__":
    main()
