import importlib.util
import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs through the C-ABI library")


def load_package():
    """Import the package directory pil2-proofman_b200/ under the module name pil2_proofman_b200."""
    name = "pil2_proofman_b200"
    if name in sys.modules:
        return sys.modules[name]
    path = os.path.join(REPO, "pil2-proofman_b200", "__init__.py")
    spec = importlib.util.spec_from_file_location(name, path,
                                                  submodule_search_locations=[os.path.dirname(path)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="session")
def pkg():
    return load_package()


@pytest.fixture(scope="session")
def orc():
    import oracle
    return oracle.Oracle()


@pytest.fixture(scope="session")
def refcpu():
    import oracle
    try:
        return oracle.RefCPU()
    except FileNotFoundError as e:
        pytest.skip("reference CPU build absent: %s" % e)


@pytest.fixture(scope="session")
def kats():
    import json
    with open(os.path.join(REPO, "tests", "golden", "reference_kats.json")) as f:
        return json.load(f)
