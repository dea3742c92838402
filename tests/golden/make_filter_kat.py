"""Writes tests/golden/filter_kat.json: the reference's filter known-answer tests
(al0vya/gpu-mwdg2 source/unittests/unit_tests_mra.cu:7-408) as inputs and expected
values, for tests/test_filter_kat.py.

The reference checks each Haar and multiwavelet filter function against the filter-bank sum
written out with its constants (source/mra/Filters.h, the active `#define NAME C(value)`
block): encode = (sum over the four children of filter x child coefficients) / 2 with
filters 0, 1, 2, 3 taking children 0, 2, 1, 3; decode = 2 x (sum over the parent's scale
coefficients and alpha, beta, gamma details of the transposed filters). Inputs are those
of the reference's tests: children 1..4 (Haar), child modes 1..12 (multiwavelet encode),
scale 1, 2, 3 and details 1..9 (decode). One reference test checks the 1y scale output
against the 1x function; here the 1y case uses the third filter rows, as the function it
names does. Tolerance 1e-6, the reference's are_reals_equal.

Run in a checkout that has the reference sources:
    python tests/golden/make_filter_kat.py <reference>/source/mra/Filters.h
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def constants(path):
    text = re.sub(r"/\*.*?\*/", "", open(path).read(), flags=re.S)
    out = {}
    for name, val in re.findall(r"^#define\s+(\w+)\s+C\(\s*([-+0-9.eE]+)\s*\)\s*$", text, flags=re.M):
        out[name] = float(val)
    return out


def main():
    k = constants(sys.argv[1])
    fmap = (0, 2, 1, 3)            # filter f acts on child fmap[f]
    # Haar: children 1, 2, 3, 4
    c = [1.0, 2.0, 3.0, 4.0]
    H0, H1, G0, G1 = k["H0"], k["H1"], k["G0"], k["G1"]
    hw = {"children": c,
          "scale": 0.5 * (H0 * (H0 * c[0] + H1 * c[2]) + H1 * (H0 * c[1] + H1 * c[3])),
          "alpha": 0.5 * (H0 * (G0 * c[0] + G1 * c[2]) + H1 * (G0 * c[1] + G1 * c[3])),
          "beta": 0.5 * (G0 * (H0 * c[0] + H1 * c[2]) + G1 * (H0 * c[1] + H1 * c[3])),
          "gamma": 0.5 * (G0 * (G0 * c[0] + G1 * c[2]) + G1 * (G0 * c[1] + G1 * c[3]))}
    # multiwavelet encode: child k has modes (0, 1x, 1y) = (3k+1, 3k+2, 3k+3); ch[m][k]
    ch = [[3.0 * kk + 1 + m for kk in range(4)] for m in range(3)]

    def analyse(tab, row):
        s = 0.0
        for f in range(4):
            for col in range(3):
                s += k[f"{tab}{f}_{row + 1}{col + 1}"] * ch[col][fmap[f]]
        return s / 2.0
    mw_enc = {"children": ch,
              "scale": [analyse("HH", r) for r in range(3)],
              "details": [[analyse(t, r) for r in range(3)] for t in ("GA", "GB", "GC")]}
    # multiwavelet decode: scale (1, 2, 3), alpha (1, 2, 3), beta (4, 5, 6), gamma (7, 8, 9)
    s = [1.0, 2.0, 3.0]
    d = [[1.0, 2.0, 3.0], [4.0, 5.0, 6.0], [7.0, 8.0, 9.0]]
    out = [[0.0] * 4 for _ in range(3)]
    for f in range(4):
        for j in range(3):
            v = 0.0
            for r in range(3):
                v += k[f"HH{f}_{r + 1}{j + 1}"] * s[r]
                for t, tab in enumerate(("GA", "GB", "GC")):
                    v += k[f"{tab}{f}_{r + 1}{j + 1}"] * d[t][r]
            out[j][fmap[f]] = 2.0 * v
    mw_dec = {"scale": s, "details": d, "children": out}
    doc = {"source": "al0vya/gpu-mwdg2 source/unittests/unit_tests_mra.cu:7-408 with the constants of "
                     "source/mra/Filters.h", "tolerance": 1e-6,
           "hw_encode": hw, "mw_encode": mw_enc, "mw_decode": mw_dec}
    with open(os.path.join(HERE, "filter_kat.json"), "w") as fp:
        json.dump(doc, fp, indent=1)
        fp.write("\n")


if __name__ == "__main__":
    main()
