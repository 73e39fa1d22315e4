"""Shared test setup: the `gpu` marker, and loaders for the product package
(directory impact-z_b200, imported as impz_b200) and the CPU oracle."""
import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def load_impz():
    if "impz_b200" in sys.modules:
        return sys.modules["impz_b200"]
    pkg = os.path.join(ROOT, "impact-z_b200")
    spec = importlib.util.spec_from_file_location(
        "impz_b200", os.path.join(pkg, "__init__.py"), submodule_search_locations=[pkg])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["impz_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def load_oracle():
    if "impz_oracle" in sys.modules:
        return sys.modules["impz_oracle"]
    spec = importlib.util.spec_from_file_location(
        "impz_oracle", os.path.join(ROOT, "oracle", "oracle.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules["impz_oracle"] = mod
    spec.loader.exec_module(mod)
    return mod


def reference_path(*parts):
    """A path inside a checkout of the reference (IMPACT-Z) named by the
    environment variable IMPZ_REFERENCE_TREE, or None when it is unset; the
    tests that read the reference's example decks or its GUI deck reader skip
    without it."""
    root = os.environ.get("IMPZ_REFERENCE_TREE")
    return os.path.join(root, *parts) if root else None


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def impz():
    return load_impz()


@pytest.fixture(scope="session")
def orc():
    return load_oracle()
