import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the CUDA library")


@pytest.fixture(scope="session")
def flop_tables():
    """Packed tables of the reference flop, made by the oracle (test infrastructure)."""
    from oracle import oracle as O
    return O.pack_flop_tables(O.REFERENCE_FLOP)
