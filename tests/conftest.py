"""pytest configuration: the `gpu` marker and the package loader.

The package directory is named `femtools.jl_b200`, which is not an importable
identifier, so it is loaded by path under the module name `femtools_b200`.
"""
import importlib.util
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def load_package():
    if "femtools_b200" in sys.modules:
        return sys.modules["femtools_b200"]
    pkg_dir = os.path.join(ROOT, "femtools.jl_b200")
    spec = importlib.util.spec_from_file_location(
        "femtools_b200", os.path.join(pkg_dir, "__init__.py"), submodule_search_locations=[pkg_dir])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["femtools_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


fem = load_package()


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libfemtools_b200")
