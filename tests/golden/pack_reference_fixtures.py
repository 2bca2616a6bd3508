"""Pack the reference's two test fixtures into reference_fixtures.tar.xz.

testsuite/atomisticPA and testsuite/hybridPA are the inputs of the reference's
own regression test (testsuite/runtests.sh:7-27, goldens at
testsuite/tests.py:10-68).  The GPU tests run them through the CUDA path on a
machine that has no copy of the reference tree, so the two directories travel
with the tests as one compressed archive, byte for byte as the reference holds
them (the tests add the `mts 0` key the current RDCONTROL.f90:485-497 requires
when they unpack).  The archive is deterministic: sorted members, fixed owner,
mode and time.

Usage:  python tests/golden/pack_reference_fixtures.py [reference tree]
        (default: $IBISCO_REFERENCE_DIR)
"""
import io
import os
import sys
import tarfile

FIXTURES = ("atomisticPA", "hybridPA")
HERE = os.path.dirname(os.path.abspath(__file__))
ARCHIVE = os.path.join(HERE, "reference_fixtures.tar.xz")


def pack(ref_dir: str, dst: str = ARCHIVE) -> str:
    with tarfile.open(dst, "w:xz", preset=9) as tar:
        for fx in FIXTURES:
            src = os.path.join(ref_dir, "testsuite", fx)
            for name in sorted(os.listdir(src)):
                path = os.path.join(src, name)
                if not os.path.isfile(path):
                    continue
                data = open(path, "rb").read()
                info = tarfile.TarInfo(f"{fx}/{name}")
                info.size = len(data)
                info.mode = 0o644
                info.mtime = 0
                info.uid = info.gid = 0
                info.uname = info.gname = ""
                tar.addfile(info, io.BytesIO(data))
    return dst


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("IBISCO_REFERENCE_DIR")
    if not ref:
        raise SystemExit("give the reference tree as an argument or in IBISCO_REFERENCE_DIR")
    print(pack(ref))
