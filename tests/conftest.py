import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

from oracle.refpath import reference_path, reference_sources  # noqa: E402

# the reference project's root (GD_REFERENCE; see oracle/refpath.py)
REFERENCE = reference_path()


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


@pytest.fixture(scope="session")
def lib():
    from geauxdock_b200 import build
    from geauxdock_b200._lib import load

    build.build()
    return load()


@pytest.fixture(scope="session")
def enepara(lib):
    from geauxdock_b200 import params

    return params.optimize_enepara(params.default_enepara0())


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import oracle as O

    if not O.ORACLE_SO.exists():
        O.build()
    return O


def have_reference_sources() -> bool:
    return reference_sources() is not None
