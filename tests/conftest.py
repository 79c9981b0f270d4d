"""Test configuration: the `gpu` marker and an importable alias for the package.

The package directory is named ``zolo-svd_b200`` (not a Python identifier), so
it is registered here as the module ``zolo_svd_b200``.
"""
import importlib.util
import os
import sys

import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def _load_pkg():
    if "zolo_svd_b200" in sys.modules:
        return sys.modules["zolo_svd_b200"]
    pkg_dir = os.path.join(ROOT, "zolo-svd_b200")
    spec = importlib.util.spec_from_file_location("zolo_svd_b200", os.path.join(pkg_dir, "__init__.py"),
                                                  submodule_search_locations=[pkg_dir])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["zolo_svd_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


_load_pkg()


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if gpu_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)
