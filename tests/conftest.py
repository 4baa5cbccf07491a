"""Shared test setup: import paths, the `gpu` marker, and the CUDA context fixture.

`-m "not gpu"` runs the oracle checks, the host-side logic (parser, LIME codec, C ABI
symbol table and error paths) and the gloo multi-rank tests; `-m gpu` runs the parity
tests of the CUDA library against the oracle through the C ABI.
"""
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
for p in (ROOT / "ecmc-qncb_b200", ROOT / "oracle", ROOT):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA library")


@pytest.fixture(scope="session")
def ctx():
    import qcb
    c = qcb.Context(0)
    yield c
    c.close()


@pytest.fixture(scope="session")
def orc():
    import oracle
    oracle.lib()
    return oracle
