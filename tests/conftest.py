"""Shared fixtures.  GPU tests carry @pytest.mark.gpu; everything else runs on CPU."""

import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
for p in (ROOT, ROOT / "quant-kernel_b200"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def qk():
    """The library under test (loads libqk_b200.so once)."""
    from quantkernel_b200 import QuantKernel

    return QuantKernel()


@pytest.fixture(scope="session")
def oracle():
    """The CPU oracle (test infrastructure)."""
    from oracle.oracle import Oracle

    return Oracle()


@pytest.fixture(scope="session")
def ref():
    """The reference library compiled from its sources, where it was built."""
    from oracle.oracle import Reference, reference_available

    if not reference_available():
        pytest.skip("oracle/_ref/libquantkernel.so not built on this machine")
    return Reference()
