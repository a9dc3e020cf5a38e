import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def _ensure_built():
    """Rebuild every native library whose sources changed since it was built
    (each library carries a digest of the sources it was built from, so a
    stale library is never tested, and a prebuilt tree whose sources match
    is used as it is)."""
    from lfric_core_b200 import build as pkg_build
    from oracle import build as oracle_build
    pkg_build.build_all()
    oracle_build.build()


_ensure_built()


@pytest.fixture(scope="session")
def ctx():
    import torch  # noqa: F401  (only to report a clear skip reason below)
    from lfric_core_b200 import lfx
    try:
        c = lfx.Context(int(os.environ.get("LFX_DEVICE", "0")))
    except Exception as e:  # pragma: no cover - GPU tests need a GPU
        pytest.fail(f"GPU context unavailable: {e}")
    yield c
    c.close()
