"""ORACLE -- load the unmodified reference modules (polyspec/base.py,
weighting.py, pspec_bin.py) from a reference checkout with the shims of
oracle/shims standing in for ducc0, healpy and pywigxjpf.  Only usable where
the reference checkout exists (the fixture generator under tests/golden runs
it there); test infrastructure only.
"""
import importlib.util
import os
import sys
import types

HERE = os.path.dirname(os.path.abspath(__file__))


def load(reference_root, modules=("base", "weighting", "pspec_bin")):
    shims = os.path.join(HERE, "shims")
    if shims not in sys.path:
        sys.path.insert(0, shims)
    root = os.path.dirname(HERE)
    if root not in sys.path:
        sys.path.insert(0, root)
    pkg_dir = os.path.join(reference_root, "polyspec")
    pkg = types.ModuleType("refpolyspec")
    pkg.__path__ = [pkg_dir]
    sys.modules["refpolyspec"] = pkg
    out = {}
    for name in modules:
        spec = importlib.util.spec_from_file_location("refpolyspec." + name, os.path.join(pkg_dir, name + ".py"))
        mod = importlib.util.module_from_spec(spec)
        sys.modules["refpolyspec." + name] = mod
        spec.loader.exec_module(mod)
        out[name] = mod
    return out
