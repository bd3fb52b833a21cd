"""Shared fixtures. GPU tests are marked ``gpu``; everything else runs on CPU."""
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an NVIDIA B200 and the built libqtrk_b200.so")
    config.addinivalue_line("markers", "slow: full-size workloads")


@pytest.fixture(scope="session")
def ref():
    """The reference CPU tracker compiled from its own sources (oracle/_ref)."""
    from oracle import RefOracle, ref_available

    if not ref_available():
        pytest.skip("oracle/_ref/libqtrk_ref.so not built (needs the reference tree; run python oracle/build.py)")
    return RefOracle()


@pytest.fixture(scope="session")
def port():
    """The FP64 restatement (oracle/qtrk_oracle.c)."""
    from oracle import PortOracle, port_available

    if not port_available():
        import subprocess

        subprocess.run([sys.executable, str(ROOT / "oracle" / "build.py")], check=True)
    return PortOracle()


@pytest.fixture(scope="session")
def qlib():
    """libqtrk_b200.so, loaded through ctypes. GPU tests fail (not skip) when it is missing."""
    from qtrk_b200 import tracker

    return tracker.load_library()
