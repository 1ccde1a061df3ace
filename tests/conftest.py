import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _build_product() -> None:
    """Builds libdynamis_cuda.so before anything imports dynamis_b200 (whose import loads it)."""
    import importlib.util

    spec = importlib.util.spec_from_file_location("_dynamis_build", ROOT / "dynamis_b200" / "build.py")
    module = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(module)
    module.build()


_build_product()


@pytest.fixture(scope="session", autouse=True)
def _built():
    from oracle import build as oracle_build

    oracle_build.build()
