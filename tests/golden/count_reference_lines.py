"""Write reference_line_counts.json: the number of lines of every reference
source file that this repository cites as `FILE:line` (Fortran sources, .inc
files, the preprocessor header, the Makefile and the test suite).  The CPU
test tests/test_citations.py checks every citation in the repository against
these counts, so it runs where the reference tree is absent.

Usage:  python tests/golden/count_reference_lines.py [reference tree]
        (default: $IBISCO_REFERENCE_DIR)
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "reference_line_counts.json")
SUFFIXES = (".f90", ".F90", ".inc", ".h", ".py", ".sh")


def count(ref: str) -> dict:
    out = {}
    for root, dirs, files in os.walk(ref):
        dirs[:] = sorted(d for d in dirs if d not in (".git", "docs"))
        for f in sorted(files):
            if f.endswith(SUFFIXES) or f == "Makefile":
                rel = os.path.relpath(os.path.join(root, f), ref)
                with open(os.path.join(root, f), "rb") as fh:
                    out[rel] = len(fh.read().splitlines())
    return out


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("IBISCO_REFERENCE_DIR")
    if not ref:
        raise SystemExit("give the reference tree as an argument or in IBISCO_REFERENCE_DIR")
    with open(OUT, "w") as f:
        json.dump(count(ref), f, indent=0, sort_keys=True)
    print(OUT)
