"""Test configuration: registers the ``gpu`` marker and makes the package importable.

The package directory ``dmrjtensor.jl_b200`` is not a valid Python identifier, so it is loaded
under the name ``dmrjtensor_b200``; the oracle (``oracle/``) is imported from the repository root.
"""
import importlib.util
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def load_package():
    if "dmrjtensor_b200" in sys.modules:
        return sys.modules["dmrjtensor_b200"]
    pkg_dir = ROOT / "dmrjtensor.jl_b200"
    spec = importlib.util.spec_from_file_location(
        "dmrjtensor_b200", pkg_dir / "__init__.py", submodule_search_locations=[str(pkg_dir)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["dmrjtensor_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def dmrgb():
    return load_package()


@pytest.fixture(scope="session")
def ctx(dmrgb):
    return dmrgb.Context(0)
