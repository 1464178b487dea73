import importlib.util
import pathlib
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def load_package():
    """Import the engine package (directory spin-glass_b200/) as spin_glass_b200."""
    if "spin_glass_b200" in sys.modules:
        return sys.modules["spin_glass_b200"]
    pkg_dir = ROOT / "spin-glass_b200"
    spec = importlib.util.spec_from_file_location(
        "spin_glass_b200", pkg_dir / "__init__.py", submodule_search_locations=[str(pkg_dir)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["spin_glass_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running statistical check")


@pytest.fixture(scope="session")
def csg():
    return load_package()


@pytest.fixture(scope="session")
def orc():
    from oracle import oracle as o
    o.build()
    return o
