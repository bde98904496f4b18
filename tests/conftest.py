import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_BUILD = os.path.join(ORACLE_DIR, "_build")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: long CPU oracle runs (set ALPINEEM_SLOW=1)")


def pytest_collection_modifyitems(config, items):
    if os.environ.get("ALPINEEM_SLOW") == "1":
        return
    skip = pytest.mark.skip(reason="long oracle run; set ALPINEEM_SLOW=1")
    for it in items:
        if "slow" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def oracle_bin():
    """Paths of the oracle executables (built from oracle/ if missing)."""
    names = ["fdtd_oracle", "fdtd_oracle_f64", "fdtd_oracle_kmax", "fdtd_oracle_kmax_f64"]
    if not all(os.path.exists(os.path.join(ORACLE_BUILD, n)) for n in names):
        subprocess.run(["make", "-s", "-C", ORACLE_DIR], check=True)
    return {n: os.path.join(ORACLE_BUILD, n) for n in names}


@pytest.fixture(scope="session")
def gpu_lib():
    """The in-tree CUDA library; a GPU test fails (not skips) if it is missing."""
    import alpineem_b200

    return alpineem_b200.load_library()
