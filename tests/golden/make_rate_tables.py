"""Build the rate-table fixtures from the reference's input files.

Source: the reference's input/rateCoef_e.csv (electron collision rates against
mean energy, 1800 rows) and input/rateCoef_i.csv (ion momentum-transfer rate),
read the way InputModule::input_BOLSIG_data does (inputModule.hpp:1413-1655),
restated by oracle.fluid.bolsig_tables -> rate_tables.npz with the eleven
BolsigVec tables and the steps dTe (K) and dEi (J); input/coefEISEE.csv read as
InputModule::input_SEE_data (inputModule.hpp:605-657), oracle.fluid.see_tables
-> see_tables.npz with the EB, RD, TS yields and dTe_SEE (K).
Usage: python <this script> <reference checkout>  (or set CATHODE_REFERENCE).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def reference_root() -> str:
    """The reference checkout: the first command-line argument, else $CATHODE_REFERENCE."""
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("CATHODE_REFERENCE")
    if not root or not os.path.isdir(root):
        sys.exit(f"usage: python {os.path.basename(__file__)} <reference checkout> (or set CATHODE_REFERENCE)")
    return root
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import fluid  # noqa: E402


def main():
    SRC = os.path.join(reference_root(), "input")
    te = open(os.path.join(SRC, "rateCoef_e.csv")).read()
    ti = open(os.path.join(SRC, "rateCoef_i.csv")).read()
    tb, dTe, dEi = fluid.bolsig_tables(te, ti)
    out = os.path.join(HERE, "rate_tables.npz")
    np.savez_compressed(out, dTe=dTe, dEi=dEi, **tb)
    print(out, {k: v.shape for k, v in tb.items()}, dTe, dEi)
    eb, rd, ts, dTe_SEE = fluid.see_tables(open(os.path.join(SRC, "coefEISEE.csv")).read())
    out = os.path.join(HERE, "see_tables.npz")
    np.savez_compressed(out, coefEISEE_eb_table=eb, coefEISEE_rd_table=rd, coefEISEE_ts_table=ts,
                        dTe_SEE=dTe_SEE)
    print(out, eb.shape, dTe_SEE)


if __name__ == "__main__":
    main()
