"""Every `FILE:line` citation of a reference source in this repository points
inside that file.

The line counts come from golden/reference_line_counts.json (written from the
reference tree by golden/count_reference_lines.py).  A citation is a reference
file name followed by a colon and a line, a range or a comma list of either
(`NONBONDED_FORCE.F90:45-104`, `VIRTUAL_DEF.f90:31,35,38`).
"""
import json
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
COUNTS = json.load(open(os.path.join(ROOT, "tests", "golden", "reference_line_counts.json")))
BY_NAME = {os.path.basename(k): v for k, v in COUNTS.items()}
SCANNED = ("ibisco_b200", "include", "oracle", "fortran", "tests", "profiles")
TOP = ("DESIGN.md", "INTEGRATION.md", "README.md", "bench.py", "__graft_entry__.py")
EXT = (".py", ".cu", ".cuh", ".cpp", ".hpp", ".h", ".f90", ".md", ".txt")
CITE = re.compile(r"([A-Za-z0-9_/]+\.(?:f90|F90|inc|h|py|sh)|Makefile):(\d+(?:-\d+)?(?:,\s?\d+(?:-\d+)?)*)")


def files():
    for d in SCANNED:
        for root, dirs, fs in os.walk(os.path.join(ROOT, d)):
            dirs[:] = [x for x in dirs if not x.startswith(("_", "."))]
            for f in fs:
                if f.endswith(EXT) and "golden" not in root:
                    yield os.path.join(root, f)
    for f in TOP:
        yield os.path.join(ROOT, f)


def citations(text):
    for m in CITE.finditer(text):
        name = os.path.basename(m.group(1))
        if name not in BY_NAME:
            continue
        for part in re.split(r",\s?", m.group(2)):
            nums = [int(x) for x in part.split("-")]
            yield name, nums, m.group(0)


def test_reference_citations_lie_inside_their_files():
    bad = []
    n = 0
    for path in files():
        text = open(path, encoding="utf-8", errors="replace").read()
        for name, nums, cite in citations(text):
            n += 1
            last = BY_NAME[name]
            if any(x < 1 or x > last for x in nums) or (len(nums) == 2 and nums[0] > nums[1]):
                bad.append(f"{os.path.relpath(path, ROOT)}: {cite} ({name} has {last} lines)")
    assert n > 100, "the scan found too few citations"
    assert not bad, "\n".join(bad)
