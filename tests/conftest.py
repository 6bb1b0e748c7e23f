"""Shared test configuration.

Markers
  gpu   needs a CUDA device (a B200); everything else runs on CPU.

The checkers (oracle/) are built on demand: the C restatement always, the
compiled reference only where QT_REFERENCE_ROOT names its source tree (a
checker built beforehand, e.g. by the package build, is used as it is).
"""

import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: test needs a CUDA GPU (B200)")


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle

    if not os.path.exists(oracle.ORACLE_SO):
        oracle.build()
    return oracle.Oracle()


@pytest.fixture(scope="session")
def reference_lib():
    import oracle

    if not oracle.reference_available():
        try:
            oracle.build(ref_root=os.environ.get("QT_REFERENCE_ROOT"))
        except Exception:
            pass
    if not oracle.reference_available():
        pytest.skip("compiled reference (oracle/_ref) not available")
    return oracle.Reference()


@pytest.fixture(scope="session")
def qt():
    import quicktex_b200

    return quicktex_b200
