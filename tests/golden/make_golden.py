"""Extract the reference test fixtures used as golden vectors.

Reads the reference checkout's ``test_data/`` (ougx/krigekit) and writes the
columns the parity tests need into this directory.  Run once in a container
that has the reference mounted:

    python tests/golden/make_golden.py /path/to/krigekit

The outputs are plain CSV files committed next to this script; nothing at
test time reads the reference checkout.
"""
import os
import sys

import pandas as pd

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref_root: str) -> None:
    td = os.path.join(ref_root, "test_data")
    # pc2d.csv: 62 observations with the reference leave-one-out column
    pd.read_csv(os.path.join(td, "pc2d.csv"))[["x", "y", "pc", "loo-cv"]].to_csv(
        os.path.join(HERE, "pc2d.csv"), index=False)
    # grid2d.csv: 4800 targets with the reference ordinary-kriging estimate/variance
    pd.read_csv(os.path.join(td, "grid2d.csv"))[["x", "y", "estimate", "variance"]].to_csv(
        os.path.join(HERE, "grid2d.csv"), index=False)
    # path4800.csv / sample4800.csv: the SGSIM visiting order and N(0, 1) draws of
    # the reference's deterministic simulation test (tests/test_sgsim.py)
    for name in ("obs_simple.csv", "grid_simple.csv", "head2d.csv", "walker.csv",
                 "gridblockpnt2d.csv", "path4800.csv", "sample4800.csv"):
        pd.read_csv(os.path.join(td, name)).to_csv(os.path.join(HERE, name), index=False)
    blk = pd.read_csv(os.path.join(td, "gridblock2d.csv"))
    blk.columns = [c.strip().lstrip("#").strip() for c in blk.columns]
    blk.to_csv(os.path.join(HERE, "gridblock2d.csv"), index=False)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path to the krigekit checkout>")
    main(sys.argv[1])
