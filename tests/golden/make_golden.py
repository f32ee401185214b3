"""Regenerate the golden fixtures of tests/golden from the reference's own tests.

Reads the reference's test sources as text (it never runs them: the
reference is Julia, which is not installed) and writes:
  philox4x32_10_kat.json  the Random123 known-answer vectors of
                          test/backends.jl:269-273 (Philox4x32-10)

Usage: python tests/golden/make_golden.py /path/to/Aeolus.jl
   or: AEOLUS_REFERENCE=/path/to/Aeolus.jl python tests/golden/make_golden.py
"""
import json
import os
import re
import sys

REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("AEOLUS_REFERENCE")
if not REF:
    sys.exit("usage: make_golden.py /path/to/Aeolus.jl (or set AEOLUS_REFERENCE)")
HERE = os.path.dirname(os.path.abspath(__file__))


def hexes(s):
    return re.findall(r"0x[0-9a-fA-F]+", s)


def philox_kats():
    src = open(os.path.join(REF, "test", "backends.jl")).read()
    lines = [l for l in src.splitlines() if "@test φ((" in l or "(0xd16cfe09" in l]
    vecs = []
    # vector 1: all-zero counter and key
    m0 = re.search(r"φ\(\(z, z, z, z\), \(z, z\)\) == \(([^)]*)\)", src)
    vecs.append({"ctr": ["0x0"] * 4, "key": ["0x0"] * 2, "out": hexes(m0.group(1))})
    m1 = re.search(r"φ\(\(f, f, f, f\), \(f, f\)\) == \(([^)]*)\)", src)
    vecs.append({"ctr": ["0xffffffff"] * 4, "key": ["0xffffffff"] * 2, "out": hexes(m1.group(1))})
    m2 = re.search(r"φ\(\((0x[^)]*)\), \((0x[^)]*)\)\) ==\s*\(([^)]*)\)", src, re.S)
    vecs.append({"ctr": hexes(m2.group(1)), "key": hexes(m2.group(2)), "out": hexes(m2.group(3))})
    assert len(lines) >= 2
    return {"source": "test/backends.jl:269-273 (Random123 kat_vectors, philox4x32_10)", "vectors": vecs}


if __name__ == "__main__":
    with open(os.path.join(HERE, "philox4x32_10_kat.json"), "w") as f:
        json.dump(philox_kats(), f, indent=1)
    print("wrote", os.path.join(HERE, "philox4x32_10_kat.json"))
