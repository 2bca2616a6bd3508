"""Source invariant of the programmatic dependent launches (CPU only).

A kernel launched with programmatic stream serialization may start while the
kernel before it in the stream still runs; it is correct only if it waits
(pdl_wait, griddepcontrol.wait) before touching memory.  Every kernel that the
host launches through launch_pdl / launch_on(..., true, ...) must therefore
open with pdl_wait(), after nothing but compile-time declarations."""
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "ibisco_b200", "csrc")


def _read(name):
    with open(os.path.join(CSRC, name)) as f:
        return f.read()


def _pdl_launched_kernels(host: str) -> set:
    names = set()
    for m in re.finditer(r"launch_pdl\(c,\s*([A-Za-z_]\w*)", host):
        names.add(m.group(1))
    for m in re.finditer(r"launch_on\(\w+,\s*true,\s*([A-Za-z_]\w*)", host):
        names.add(m.group(1))
    if "nb_kernel" in names:  # the nonbonded launch goes through nb_kernel<R, B>()
        names.discard("nb_kernel")
        names.update({"k_nonbonded", "k_nonbonded_f32"})
    return names


def _body_opening(kernels: str, name: str) -> list:
    m = re.search(r"__global__ void (?:__launch_bounds__\([^)]*\) )?%s\(" % name, kernels)
    assert m, f"kernel {name} not found"
    body = kernels[kernels.index("{\n", m.end()) + 2:]
    lines = []
    for line in body.splitlines():
        line = line.strip()
        if not line or line.startswith("//"):
            continue
        lines.append(line)
        if line.startswith("pdl_wait();") or len(lines) > 4:
            break
    return lines


def test_every_programmatic_launch_waits_first():
    host = _read("ibg_device.cu")
    kernels = _read("ibg_kernels.cuh")
    names = _pdl_launched_kernels(host)
    # the chain of one step and of a batch step
    assert {"k_nonbonded_f32", "k_nb_near", "k_nb_collect", "k_finalize", "k_list_build_warp",
            "k_list_build_thread"} <= names
    for name in sorted(names):
        opening = _body_opening(kernels, name)
        assert opening and opening[-1] == "pdl_wait();", (name, opening)
        for line in opening[:-1]:
            assert line.startswith(("using ", "constexpr ")), (name, line)
