import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))

from ref import REFERENCE_DIR  # noqa: E402  (oracle/ref.py)

REFERENCE_SRC = os.path.join(REFERENCE_DIR, "src")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


@pytest.fixture(scope="session")
def oracle_built():
    """Build the FP64 restatement (always) and the shim-hosted reference
    (only where the reference tree exists)."""
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
    if os.path.isdir(REFERENCE_SRC):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref", f"REF={REFERENCE_DIR}"], check=True)
    return True


@pytest.fixture(scope="session")
def gpu_lib():
    from awsemmd_b200 import build

    build.build()
    from awsemmd_b200 import engine

    return engine.load_library()


def neigh_of(g):
    """(skin, delay, every, check) of a golden case's runs: LAMMPS's defaults
    unless the case was made with other neighbour settings."""
    if "neigh" not in g.files:
        return 2.0, 0, 1, 1
    skin, delay, every, check = (float(v) for v in g["neigh"])
    return skin, int(delay), int(every), int(check)


def write_case(name, tmp_path):
    """Write a golden case's inputs and check they regenerate byte for byte."""
    import numpy as np
    import make_golden

    files = make_golden.write_case(name, str(tmp_path / name))
    g = np.load(os.path.join(ROOT, "tests", "golden", f"{name}.npz"))
    assert make_golden.dir_hash(files["workdir"]) == str(g["inputs_sha256"]), \
        f"{name}: regenerated inputs differ from the ones the golden vectors were made from"
    return files, g
