"""Test configuration: the `gpu` marker, and the package/oracle import paths.

The product package lives in the directory `h2factory.jl_b200/`; it is registered here under the
import name `h2factory_b200`. The oracle (test infrastructure) is imported as `oracle.oracle`.
"""

import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "h2factory.jl_b200")


def _register_package():
    if "h2factory_b200" in sys.modules:
        return
    spec = importlib.util.spec_from_file_location(
        "h2factory_b200", os.path.join(PKG_DIR, "__init__.py"),
        submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["h2factory_b200"] = mod
    spec.loader.exec_module(mod)


_register_package()
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
TESTS = os.path.dirname(os.path.abspath(__file__))
if TESTS not in sys.path:
    sys.path.insert(0, TESTS)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")


def pytest_collection_modifyitems(config, items):
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:  # pragma: no cover
        has_gpu = False
    if has_gpu:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)
