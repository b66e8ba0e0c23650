import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(1, os.path.join(ROOT, "oracle"))  # screen_ref (numpy reference of the screen network)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running CPU test")


def load_package():
    """Import the product package from its directory (its name is not a Python identifier)."""
    if "turbogap_b200" in sys.modules:
        return sys.modules["turbogap_b200"]
    pkg_dir = os.path.join(ROOT, "turbogap_2.0_b200")
    spec = importlib.util.spec_from_file_location(
        "turbogap_b200", os.path.join(pkg_dir, "__init__.py"), submodule_search_locations=[pkg_dir])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["turbogap_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="session")
def tg():
    return load_package()


@pytest.fixture(scope="session")
def synth(tg):
    return tg.synth


@pytest.fixture(scope="session")
def orc():
    import oracle_lib
    oracle_lib.lib()
    return oracle_lib
