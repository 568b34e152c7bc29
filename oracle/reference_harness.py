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


def load_cython(reference_root=None):
    """Register the reference's Cython modules under ``refpolyspec.cython``: the
    compiled tauNL_utils and ideal_fisher of oracle/_ref (built by
    oracle/build_ref.sh from the reference sources) and the numpy k_integrals shim
    (GSL, which the compiled module needs, is absent).  Call before loading
    tspec_template."""
    import importlib.machinery
    if "refpolyspec" not in sys.modules:
        raise RuntimeError("load() the reference package first")
    cy = types.ModuleType("refpolyspec.cython")
    cy.__path__ = []
    sys.modules["refpolyspec.cython"] = cy
    ref_dir = os.path.join(HERE, "_ref")
    suffix = importlib.machinery.EXTENSION_SUFFIXES[0]
    for name in ("tauNL_utils", "ideal_fisher"):
        path = os.path.join(ref_dir, name + suffix)
        if not os.path.exists(path):
            raise RuntimeError("compiled reference module %s missing: run oracle/build_ref.sh" % path)
        spec = importlib.util.spec_from_file_location("refpolyspec.cython." + name, path)
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        sys.modules["refpolyspec.cython." + name] = mod
    shims = os.path.join(HERE, "shims")
    spec = importlib.util.spec_from_file_location("refpolyspec.cython.k_integrals", os.path.join(shims, "k_integrals.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    sys.modules["refpolyspec.cython.k_integrals"] = mod
