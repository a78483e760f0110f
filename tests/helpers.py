"""Import helpers shared by the tests: the package (directory name has a hyphen) and the oracle."""
import importlib.util
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _load(name, path):
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


pkg = _load("pi_compute_b200", os.path.join(ROOT, "pi-compute_b200", "__init__.py"))
oracle = _load("pi_oracle", os.path.join(ROOT, "oracle", "oracle.py"))
GOLDEN = os.path.join(ROOT, "tests", "golden")
