"""Extract the reference's own golden vectors into reference_goldens.json.

The reference test suite (testsuite/tests.py:10-68) pins, for its two
fixtures, the coordinates (Angstrom) and velocities (Angstrom/ps) of the first
three atoms and the box after 10 and 40 steps.  This script reads that file
as text (it is not imported: it needs MDAnalysis and nose) and writes the
numbers as JSON so the oracle tests do not depend on the reference tree.

Usage:  python tests/golden/extract_goldens.py [path/to/testsuite/tests.py]
        (default: testsuite/tests.py under $IBISCO_REFERENCE_DIR)
"""
import ast
import json
import os
import re
import sys



def extract(path: str) -> dict:
    src = open(path).read()
    out = {}
    for cls, key in (("reference_hybrid_data", "hybridPA"), ("reference_atomistic_data", "atomisticPA")):
        m = re.search(r"class %s\(object\):(.*?)(?=\nclass |\Z)" % cls, src, re.S)
        body = m.group(1)
        rec = {}
        for name in ("ref_coords_short", "ref_velos_short", "ref_box_short", "ref_coords_long", "ref_velos_long",
                     "ref_box_long"):
            mm = re.search(name + r"\s*=\s*np\.array\((\[.*?\])\s*,\s*(?:#[^\n]*\n\s*)?dtype", body, re.S)
            txt = re.sub(r"#[^\n]*", "", mm.group(1))
            rec[name] = ast.literal_eval(txt)
        out[key] = rec
    return out


if __name__ == "__main__":
    if len(sys.argv) > 1:
        path = sys.argv[1]
    elif os.environ.get("IBISCO_REFERENCE_DIR"):
        path = os.path.join(os.environ["IBISCO_REFERENCE_DIR"], "testsuite", "tests.py")
    else:
        raise SystemExit("give testsuite/tests.py as an argument or the reference tree in IBISCO_REFERENCE_DIR")
    data = extract(path)
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_goldens.json")
    with open(dst, "w") as f:
        json.dump({"source": "testsuite/tests.py:10-68", "units": {"coords": "Angstrom", "velocities": "Angstrom/ps"},
                   "frames": {"short": 10, "long": 40}, **data}, f, indent=1)
    print(dst)
