"""pytest configuration: the ``gpu`` marker and shared helpers on sys.path."""

import pathlib
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
for p in (ROOT, ROOT / "tests"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config: pytest.Config) -> None:
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); calls the CUDA kernels")
    config.addinivalue_line("markers", "slow: full-size checks that take tens of seconds")


@pytest.fixture(scope="session", autouse=True)
def _built_libraries() -> None:
    """Make sure the CUDA library and the oracles are built (no-op when current)."""
    from aprict_b200 import build

    build.build()
    from oracle import oracle

    if not oracle.ORACLE_SO.exists() or not oracle.have_ref():
        oracle.build()  # make: builds what is missing; the reference-compiled part only where its sources exist
