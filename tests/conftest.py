import os
import sys

import numpy as np
import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
GOLDEN = os.path.join(ROOT, "tests", "golden")
from refpath import REF_DATA  # noqa: E402


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200 / sm_100a)")


def have_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def mech_dir(tmp_path_factory):
    return str(tmp_path_factory.mktemp("mechs"))


_generated = {}


def synth(name, directory):
    """Write (once per session) the seeded synthetic mechanism `name`."""
    if name not in _generated:
        from zerork_b200 import mechgen
        g = mechgen.generate(mechgen.SPECS[name])
        _generated[name] = (g, g.write(directory))
    return _generated[name]


@pytest.fixture(scope="session")
def c1(mech_dir):
    return synth("c1_h2", mech_dir)


@pytest.fixture(scope="session")
def c2(mech_dir):
    return synth("c2_53", mech_dir)


@pytest.fixture(scope="session")
def c3(mech_dir):
    return synth("c3_160", mech_dir)


def golden(name):
    return dict(np.load(os.path.join(GOLDEN, f"ref_{name}.npz"), allow_pickle=False))


def ref_built():
    import zrk_oracle as zo
    return zo.ref_available("libc") and os.path.isdir(REF_DATA)


def oracle_tables(pm):
    """Oracle tables fed with the product loader's tables (pinned bit-exact to
    the reference's own by tests/test_loader.py)."""
    import zrk_oracle as zo
    return zo.OracleTables(zo.with_counts(pm.tables()))


def scaled_err(a, b, scale, floor=1e-300):
    """max |a-b| / scale over entries (scale = rounding-error magnitude)."""
    a, b, scale = np.asarray(a), np.asarray(b), np.asarray(scale)
    d = np.abs(a - b)
    return float(np.max(d / np.maximum(scale, floor))) if d.size else 0.0
