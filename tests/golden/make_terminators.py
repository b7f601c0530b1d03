"""Extract the golden complex chains of asr's terminator test into terminators.json.

Reads ``test/test_terminators.f90`` of the reference checkout given on the command line (read as text, nothing is
executed) and writes the two 24-level Cr e_g chains ``cr1`` / ``cr2`` (columns Re a, Im a, Re b, Im b), their energies
``zc1`` / ``zc2`` (lines 25-76) and the six-level real chain of its test 6 (line 128).  The fixture is committed; this
script documents where every number comes from.

usage: python tests/golden/make_terminators.py <asr checkout> [out.json]
"""
import json
import os
import re
import sys


def _floats(text):
    return [float(x.replace("_dp", "").replace("d", "e")) for x in re.findall(r"[-+]?\d+\.\d+e[-+]\d+_dp", text)]


def main():
    root = sys.argv[1]
    out = sys.argv[2] if len(sys.argv) > 2 else os.path.join(os.path.dirname(os.path.abspath(__file__)), "terminators.json")
    src = open(os.path.join(root, "test", "test_terminators.f90")).read()
    res = {"source": "test/test_terminators.f90"}
    for name in ("cr1", "cr2"):
        m = re.search(name + r"\(4, 24\) = reshape\(\[(.*?)\], \[4, 24\]\)", src, re.S)
        vals = _floats(m.group(1))
        assert len(vals) == 96, (name, len(vals))
        res[name] = {"re_a": vals[0::4], "im_a": vals[1::4], "re_b": vals[2::4], "im_b": vals[3::4]}
    m = re.search(r"zc1 = cmplx\(([^,]+), ([^,]+), dp\), &\s*zc2 = cmplx\(([^,]+), ([^,]+), dp\)", src)
    z = [float(m.group(k).replace("_dp", "")) for k in range(1, 5)]
    res["zc1"] = [z[0], z[1]]
    res["zc2"] = [z[2], z[3]]
    m = re.search(r"a\(1:6\) = \[([^\]]+)\]; b\(1:6\) = \[([^\]]+)\]", src)
    res["chain6_a"] = [float(x.strip().replace("_dp", "")) for x in m.group(1).split(",")]
    res["chain6_b"] = [float(x.strip().replace("_dp", "")) for x in m.group(2).split(",")]
    res["test6_energies"] = {"re_start": -2.4, "re_step": 0.6, "count": 9, "im": 0.05}
    res["expect"] = {"hull_ratio_below": 1.0, "bp_ratio_above": 1.0, "bp_vs_asymptote_tol": 1.0e-10,
                     "bp_uniform_n": 56, "bp_uniform_tol": 1.0e-2}
    with open(out, "w") as f:
        json.dump(res, f, indent=1)
    print("wrote", out)


if __name__ == "__main__":
    main()
