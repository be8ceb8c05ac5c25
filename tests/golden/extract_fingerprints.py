"""Extract the reference's golden fingerprints into reference_fingerprints.json.

The numbers were produced by external codes (Bridge++ 2.1.3 and SIMULATeQCD
767a1b1) and pasted into LatticeMatrices.jl's own tests.  This script reads
those test files as text and records each tuple with its file:line so that
the committed fixture can be traced back.  It only runs in a checkout that has
the reference tree; the fixture it writes is committed.

    python tests/golden/extract_fingerprints.py /path/to/LatticeMatrices.jl
"""
import json
import os
import re
import sys

NUM = r"[-+]?\d+\.\d+(?:[eE][-+]?\d+)?"


def _tuples(text):
    return [[float(v) for v in re.findall(NUM, t)]
            for t in re.findall(r"\(\s*(" + NUM + r"(?:\s*,\s*" + NUM +
                                r")*\s*,?)\s*\)", text)]


def _line_of(src, needle):
    return src[: src.index(needle)].count("\n") + 1


def main(root):
    out = {}
    # Bridge++ staggered D / D^dagger on 4x2x2x2 (test/staggered_dirac.jl)
    path = os.path.join(root, "test", "staggered_dirac.jl")
    src = open(path).read()
    block = src[src.index("expected = (\n                D="):]
    block = block[: block.index("for (mode")]
    d_part = block[block.index("D=("): block.index("Ddag=(")]
    g_part = block[block.index("Ddag=("):]
    out["bridgepp_staggered"] = {
        "source": "test/staggered_dirac.jl:%d" % _line_of(src, "D=(-32.4"),
        "lattice": [4, 2, 2, 2], "mass": 0.17, "phases": [1, 1, 1, -1],
        "links": "_staggered_test_links", "psi": "_staggered_test_fermion",
        "rtol": 2e-13, "atol": 8e-10,
        "D": [float(v) for v in re.findall(NUM, d_part)],
        "Ddag": [float(v) for v in re.findall(NUM, g_part)],
    }

    # SIMULATeQCD level-1 Fat7 on 4^4 (test/hisq_smearing.jl)
    path = os.path.join(root, "test", "hisq_smearing.jl")
    src = open(path).read()
    start = src.index("expected = (", src.index("SIMULATeQCD level-1"))
    block = src[start: src.index("if rank == 0", start)]
    out["simulateqcd_level1_fat7"] = {
        "source": "test/hisq_smearing.jl:%d" % _line_of(src, block),
        "lattice": [4, 4, 4, 4], "links": "_staggered_test_links",
        "rtol": 2e-14, "atol": 5e-7,
        "expected": _tuples(block[block.index("(") + 1:]),
    }

    # SIMULATeQCD complete HISQ fat + Naik on 4^4 (test/hisq_full_smearing.jl)
    path = os.path.join(root, "test", "hisq_full_smearing.jl")
    src = open(path).read()
    fat0 = src.index("expected_fat = (")
    long0 = src.index("expected_long = (")
    end = src.index("for mu in 1:4", long0)
    fat = src[fat0 + len("expected_fat = ("): long0]
    lng = src[long0 + len("expected_long = ("): end]
    out["simulateqcd_full_hisq"] = {
        "source": "test/hisq_full_smearing.jl:%d" % _line_of(
            src, "expected_fat = ("),
        "lattice": [4, 4, 4, 4], "naik_epsilon": -0.083,
        "links": "_staggered_test_links * 0.05 + identity",
        "rtol": 3e-14, "atol": 2e-8,
        "fat": _tuples(fat), "long": _tuples(lng),
    }
    for key, val in out.items():
        for name in ("D", "Ddag"):
            if name in val:
                assert len(val[name]) == 5, (key, name)
        for name in ("expected", "fat", "long"):
            if name in val:
                assert len(val[name]) == 4 and all(
                    len(t) == 5 for t in val[name]), (key, name, val[name])
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)),
                       "reference_fingerprints.json")
    with open(dst, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", dst)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/extract_fingerprints.py /path/to/LatticeMatrices.jl")
    main(sys.argv[1])
