import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
HERE = os.path.dirname(os.path.abspath(__file__))
if HERE not in sys.path:
    sys.path.insert(0, HERE)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle

    oracle.lib()
    return oracle


@pytest.fixture(scope="session")
def ref_cn(oracle_mod):
    """The reference's own _cn code (oracle/_ref); built here when the
    reference tree is present, skipped where it is neither built nor
    buildable."""
    if not oracle_mod.ref_available():
        try:
            oracle_mod.build()
        except Exception:
            pass
    if not oracle_mod.ref_available():
        pytest.skip("oracle/_ref (reference _cn build) not available")
    return oracle_mod
