"""Generates the golden fixtures of tests/golden/.

reference_kats.json  known-answer tests of the reference's own test file
                     src/tests/test_photon_prob.jl (values transcribed with
                     their file:line) and the Random123 Philox4x32-10
                     and Philox2x32-10 known-answer vectors (the algorithms
                     the kernels and the oracle share).
oracle_golden.json   outputs of the FP64 oracle on small fixed cases (medium
                     spot values, Cherenkov knots, a reference-compatible run
                     and a physical-mode run), so that any change to the
                     oracle's arithmetic shows up as a failing CPU test.

Run from the repository root: python tests/golden/make_golden.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from oracle import oracle as O  # noqa: E402
from oracle import tables as tb  # noqa: E402

REFERENCE_KATS = {
    "source": "src/tests/test_photon_prob.jl",
    "uniform_range": {"line": "13-17", "a": 2.0, "b": 5.0, "n": 10000},
    "hg_mean": {"line": "19-21", "g": 0.97, "n": 100000, "expected_mean": 0.97, "atol": 0.01},
    "rotate_identity": {"line": "26-28", "old": [0.0, 0.0, 1.0], "new": [0.0, 1.0, 0.0],
                        "expected": [0.0, 1.0, 0.0]},
    "rotate_flip": {"line": "29-30", "old": [0.0, 0.0, -1.0], "new": [0.0, 1.0, 0.0],
                    "expected": [0.0, -1.0, 0.0]},
    "rotate_y_to_minus_z": {"line": "37-41", "old": [0.0, 1.0, 0.0], "new": [0.0, 1.0, 0.0],
                            "expected": [0.0, 0.0, -1.0]},
    "rotate_unit_norm": {"line": "43-53", "old": [0.2, 0.3, 1.0], "new": [-5.0, 1.0, -20.0]},
    "rotate_vs_rodrigues": {"line": "55-64", "old": [0.2, 0.3, 1.0], "g": 0.97},
    "position_update": {"line": "67-73", "pos": [0.0, 0.0, 0.0], "dir": [0.0, 1.0, 0.0], "step": 10.0,
                        "expected": [0.0, 10.0, 0.0]},
    "interp_sorted": {"line": "75-85", "xs": [0.0, 1.0, 2.0, 3.0, 4.0], "ys": [0.0, 1.0, 4.0, 9.0, 16.0],
                      "cases": [[0.5, 0.5], [1.5, 2.5], [4.5, 16.0], [-1.0, 0.0]]},
    "interp_equidistant": {"line": "86-89", "knots": [0.0, 1.0, 4.0, 9.0, 16.0], "lower": 0.0, "upper": 4.0,
                           "cases": [[0.5, 0.5], [1.5, 2.5], [4.5, 16.0], [-1.0, 0.0]]},
}

# Random123 kat_vectors, philox4x32 R=10: (counter[4], key[2]) -> out[4]
PHILOX_KATS = [
    {"ctr": [0, 0, 0, 0], "key": [0, 0], "out": [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]},
    {"ctr": [0xffffffff] * 4, "key": [0xffffffff] * 2,
     "out": [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]},
    {"ctr": [0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344], "key": [0xa4093822, 0x299f31d0],
     "out": [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]},
]

# Random123 kat_vectors, philox2x32 R=10: (counter[2], key) -> out[2]
PHILOX2_KATS = [
    {"ctr": [0, 0], "key": 0, "out": [0xff1dae59, 0x6cd10df2]},
    {"ctr": [0xffffffff, 0xffffffff], "key": 0xffffffff, "out": [0x2c3f628b, 0xab4fd7ad]},
    {"ctr": [0x243f6a88, 0x85a308d3], "key": 0x13198a2e, "out": [0xdd7ce038, 0xf62a4c12]},
]


def hits_to_list(h, k):
    rows = []
    for r in h[:k]:
        rows.append({"pair": int(r["pair"]), "photon": int(r["photon"]), "step": int(r["step"]),
                     "pos": [float(x) for x in r["pos"]], "dir0": [float(x) for x in r["dir0"]],
                     "dir": [float(x) for x in r["dir"]], "time": float(r["time"]),
                     "weight": float(r["weight"]), "wavelength": float(r["wavelength"]),
                     "dist": float(r["dist"])})
    return rows


def oracle_golden():
    m = tb.cascadia(35.0, 2.0)
    wls = [300.0, 350.0, 400.0, 450.0, 500.0, 550.0, 600.0, 650.0, 700.0, 750.0, 800.0]
    knots = tb.cherenkov_spectrum_knots((300.0, 800.0), 20, m)
    pmt = tb.load_pmt_table(os.path.join(REPO, "photonprop.jl_b200", "photonprop_b200", "data",
                                         "pmt_acceptance.csv"))
    T = O.make_tables(m, knots, pmt=pmt)
    out = {"medium": {"salinity": m.salinity, "pressure_atm": m.pressure, "temperature": m.temperature,
                      "c_small": m.vol_conc_small_part, "c_large": m.vol_conc_large_part},
           "wavelengths": wls,
           "refractive_index": [float(x) for x in tb.refractive_index(wls, m)],
           "group_index": [float(x) for x in tb.group_index(wls, m)],
           "scattering_length": [float(x) for x in tb.scattering_length(wls, m)],
           "absorption_length": [float(x) for x in tb.absorption_length(wls)],
           "pmt_acceptance": [float(x) for x in tb.pmt_acceptance(wls, pmt)],
           "cherenkov_knots_20": [float(x) for x in knots]}
    # reference-compatible run: propagate_distance geometry (sphere on +z)
    p = O.pairs_array(1)
    p[0]["target"] = (0.0, 0.0, 10.0)
    p[0]["radius"] = 0.21
    p[0]["n_photons"] = 20000
    p[0]["seed"] = 0
    o = O.make_opts(mode=O.MODE_COMPAT, g=0.99, hist_bins=0)
    h, s, _, steps, total = O.propagate(T, p, o, n_threads=1)
    out["compat_run"] = {"pair": {"target": [0.0, 0.0, 10.0], "radius": 0.21, "n_photons": 20000, "seed": 0},
                         "g": 0.99, "n_hits": int(total), "steps": int(steps),
                         "stats": [float(x) for x in s[0]], "first_hits": hits_to_list(h, 25)}
    # physical-mode run: isotropic source, sphere at +x 10 m, 500 x 1 ns bins
    p = O.pairs_array(1)
    p[0]["target"] = (10.0, 0.0, 0.0)
    p[0]["radius"] = 0.21
    p[0]["n_photons"] = 100000
    p[0]["seed"] = 0
    o = O.make_opts(mode=O.MODE_PHYSICAL, g=0.95, t_max=500.0, hist_bins=500, flags=O.OPT_PMT_WEIGHT)
    h, s, hist, steps, total = O.propagate(T, p, o, n_threads=1)
    out["physical_run"] = {"pair": {"target": [10.0, 0.0, 0.0], "radius": 0.21, "n_photons": 100000, "seed": 0},
                           "g": 0.95, "t_max": 500.0, "n_hits": int(total), "steps": int(steps),
                           "stats": [float(x) for x in s[0]],
                           "hist_nonzero": [[int(i), float(hist[0, i])] for i in np.nonzero(hist[0])[0]],
                           "hits": hits_to_list(h, len(h))}
    return out


def main():
    with open(os.path.join(HERE, "reference_kats.json"), "w") as f:
        json.dump({"reference": REFERENCE_KATS, "philox4x32_10": PHILOX_KATS, "philox2x32_10": PHILOX2_KATS}, f,
                  indent=1)
    with open(os.path.join(HERE, "oracle_golden.json"), "w") as f:
        json.dump(oracle_golden(), f, indent=1)


if __name__ == "__main__":
    main()
