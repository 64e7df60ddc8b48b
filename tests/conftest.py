import importlib
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))
TESTS = Path(__file__).resolve().parent
if str(TESTS) not in sys.path:
    sys.path.insert(0, str(TESTS))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def cfsb():
    """The engine's Python binding (package folder name starts with a digit)."""
    pkg = importlib.import_module("2d_compressible_flow_solver_b200")
    if not pkg.LIB_PATH.exists():
        importlib.import_module("2d_compressible_flow_solver_b200.build").build()
    pkg.load_library()
    return pkg


@pytest.fixture(scope="session")
def workloads():
    return importlib.import_module("2d_compressible_flow_solver_b200.workloads")
