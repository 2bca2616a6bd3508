import os
import shutil
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

# The reference's own test fixtures (testsuite/atomisticPA, testsuite/hybridPA)
# travel with the tests as golden/reference_fixtures.tar.xz (made by
# golden/pack_reference_fixtures.py), so they run wherever the tests run.
FIXTURE_ARCHIVE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_fixtures.tar.xz")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs on a B200)")


def reference_fixture(tmp_root: str, name: str) -> str:
    """Unpack a reference test fixture and add the `mts 0` key that the current
    RDCONTROL.f90:485-497 requires (the fixtures predate it)."""
    import tarfile

    dst = os.path.join(tmp_root, name)
    if not os.path.isdir(dst):
        with tarfile.open(FIXTURE_ARCHIVE) as tar:
            members = [m for m in tar.getmembers() if m.name.startswith(name + "/") and m.isfile()]
            if not members:
                pytest.skip(f"fixture {name} not in the archive")
            tar.extractall(tmp_root, members=members, filter="data")
        ctl = os.path.join(dst, "control")
        lines = [l for l in open(ctl).read().splitlines() if l.strip() not in ("end", "END", "End")]
        lines += ["mts                        0", "end"]
        open(ctl, "w").write("\n".join(lines) + "\n")
    return dst


def with_control(spec, **keys):
    """The spec with some control-file keys replaced."""
    spec.control = dict(spec.control, **keys)
    return spec


@pytest.fixture(scope="session")
def sysdir(tmp_path_factory):
    """Factory: name -> directory of a seeded synthetic system (built once)."""
    from ibisco_b200 import synth

    base = tmp_path_factory.mktemp("systems")
    made = {}
    builders = {
        "fluid": lambda: synth.lj_fluid(n=1500, seed=11, nsteps=50, dmin=0.42),
        "fluid_sf": lambda: synth.lj_fluid(n=1500, seed=11, nsteps=2000, dmin=0.42, shifted=True, dt=0.005),
        "melt": lambda: synth.polymer_melt(nchains=24, nper=40, seed=12, nsteps=50),
        "mix4": lambda: synth.feature_mix(seed=7, non_bonded=4),
        "mix5_mts": lambda: synth.feature_mix(seed=8, non_bonded=5, nmts=3),
        "mix_npt": lambda: synth.feature_mix(seed=9, ensemble="NPT"),
        "mix_nve": lambda: synth.feature_mix(seed=10, ensemble="NVE"),
        "hybrid": lambda: synth.hybrid_melt(n_atomistic=32, n_cg=32, nmono=20, seed=13, nsteps=100),
        # initialize_velocities Y: SCALEV rescales the file's velocities (drawn
        # at 400 K) to the control file's 350 K
        "mix_y": lambda: with_control(synth.feature_mix(seed=15), initialize_velocities="Y", temperature=350),
        # 3x3x3 cells of ~220 particles: ~3,100 list candidates per cell
        "dense": lambda: synth.lj_fluid(n=6000, rho=45.0, seed=14, nsteps=10, dmin=0.12),
    }

    def get(name):
        if name not in made:
            d = str(base / name)
            synth.write_system(builders[name](), d)
            made[name] = d
        return made[name]

    return get


@pytest.fixture(scope="session")
def reftree(tmp_path_factory):
    base = str(tmp_path_factory.mktemp("reference_fixtures"))
    return lambda name: reference_fixture(base, name)


def rel_maxnorm(a, b):
    a = np.asarray(a, float)
    b = np.asarray(b, float)
    den = np.abs(b).max()
    return float(np.abs(a - b).max() / den) if den > 0 else float(np.abs(a - b).max())
