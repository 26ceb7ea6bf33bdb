"""Shared fixtures.  GPU tests carry @pytest.mark.gpu; the rest run on CPU."""
import importlib.util
import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, GOLDEN)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


def _load_package():
    if "acc_gp_b200" in sys.modules:
        return sys.modules["acc_gp_b200"]
    pkg = os.path.join(ROOT, "acc-gp_b200")
    spec = importlib.util.spec_from_file_location("acc_gp_b200", os.path.join(pkg, "__init__.py"),
                                                  submodule_search_locations=[pkg])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["acc_gp_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="session")
def gp():
    return _load_package()


@pytest.fixture(scope="session")
def oracle():
    import oracle as orc
    return orc


@pytest.fixture(scope="session")
def cases():
    from cases import CASES, build_case
    return CASES, build_case


def golden(name):
    with open(os.path.join(GOLDEN, f"{name}.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def ctx(gp):
    c = gp.Context(0)
    yield c
    c.close()
