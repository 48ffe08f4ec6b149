"""Shared pytest set-up: the ``gpu`` marker, import paths and common fixtures."""
import importlib.util
import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running CPU test")


def load_package():
    """Imports ``special-topics_b200/`` (a folder name Python cannot import directly)."""
    name = "special_topics_b200"
    if name in sys.modules:
        return sys.modules[name]
    pkg_dir = os.path.join(ROOT, "special-topics_b200")
    spec = importlib.util.spec_from_file_location(name, os.path.join(pkg_dir, "__init__.py"),
                                                  submodule_search_locations=[pkg_dir])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def load_scenario(name):
    with open(os.path.join(GOLDEN, "scenarios", name + ".json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def golden_out():
    with open(os.path.join(GOLDEN, "ref_out_ifa_fr4_200.json")) as f:
        return json.load(f)
