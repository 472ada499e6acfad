"""Regenerates the package's PMT data tables from a PhotonProp.jl checkout
(a maintenance script, not part of the product).

pmt_acceptance.csv: the PMT quantum-efficiency curve of PhotonProp.jl
(PMTAcc.csv, read at module load by src/detection.jl:31-33), unchanged
values, written with a header.  pmt_acceptance_5nm.csv: the same curve
linearly interpolated at 5 nm from 300 to 700 nm (81 entries), the
tabulation the one-pair-per-launch cone workload uses.

Usage: python tests/golden/make_pmt_data.py /path/to/PhotonProp.jl
"""
import os
import sys

import numpy as np

HERE = os.path.join(os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))),
                    "photonprop.jl_b200", "photonprop_b200", "data")


def main(ref):
    d = np.loadtxt(os.path.join(ref, "PMTAcc.csv"), delimiter=",")
    with open(os.path.join(HERE, "pmt_acceptance.csv"), "w") as f:
        f.write("# wavelength_nm,acceptance  (PhotonProp.jl PMTAcc.csv)\n")
        for wl, acc in d:
            f.write(f"{float(wl)!r},{float(acc)!r}\n")
    grid = np.arange(300.0, 700.0 + 0.5, 5.0)
    acc5 = np.interp(grid, d[:, 0], d[:, 1])
    with open(os.path.join(HERE, "pmt_acceptance_5nm.csv"), "w") as f:
        f.write("# wavelength_nm,acceptance  (PMTAcc.csv interpolated at 5 nm, 300-700 nm)\n")
        for wl, acc in zip(grid, acc5):
            f.write(f"{float(wl)!r},{float(acc)!r}\n")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_pmt_data.py <PhotonProp.jl checkout>")
    main(sys.argv[1])
