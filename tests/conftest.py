"""Shared test set-up: the `gpu` marker, the package loader (the package
directory is named croma-fp_b200, which is not an importable identifier),
and the checker modules under oracle/."""
import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def load_package():
    if "croma_fp_b200" in sys.modules:
        return sys.modules["croma_fp_b200"]
    pkg_dir = os.path.join(ROOT, "croma-fp_b200")
    spec = importlib.util.spec_from_file_location(
        "croma_fp_b200", os.path.join(pkg_dir, "__init__.py"),
        submodule_search_locations=[pkg_dir])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["croma_fp_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


load_package()


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
