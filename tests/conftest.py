import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")
    config.addinivalue_line("markers", "slow: large CPU-side case")


@pytest.fixture(scope="session", autouse=True)
def _built_libraries():
    """Builds libclspmv_b200.so and the oracle libraries once per session."""
    from clspmv_mic_b200 import build as B
    from oracle import oracle as O
    if not os.environ.get("CLSPMV_SKIP_BUILD"):
        if B.LIB.exists() or os.environ.get("CLSPMV_BUILD", "1") == "1":
            try:
                B.build()
            except Exception:
                if not B.LIB.exists():
                    raise
        if not O.PORT_LIB.exists() or O.REFERENCE_TREE.exists():
            O.build(ref=True)
    yield


def ref_or_skip():
    from oracle import oracle as O
    L = O.ref()
    if L is None:
        pytest.skip("compiled reference (oracle/_ref) not available here")
    return L
