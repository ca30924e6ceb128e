import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU (B200) and libdfcuda.so")
    config.addinivalue_line("markers", "slow: larger CPU cases")


def _have_gpu() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _have_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Builds the library and the oracle in tree when sources changed."""
    from dataframe_mojo_b200.build import build_library, build_oracle

    build_oracle()
    if os.environ.get("DFC_SKIP_BUILD") != "1":
        try:
            build_library()
        except RuntimeError as e:  # no nvcc: GPU tests fail loudly on the missing library
            print(f"libdfcuda.so build skipped: {e}", file=sys.stderr)
    yield
