"""The C ABI library loads and exports every function include/zsme.h
declares (no compute call: runs without a GPU)."""
import ctypes
import os
import re

from zoomy_dmplex_b200 import native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    names = []
    for fn in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if fn.endswith(".h"):
            src = open(os.path.join(ROOT, "include", fn)).read()
            names += re.findall(r"^\s*(?:const\s+)?[\w\*\s]+?\b(zsme_\w+)\s*\(", src, re.M)
    return sorted(set(names))


def test_library_exports_header():
    lib = native.load()
    names = declared()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n


def test_models_registered():
    names = native.model_names()
    assert {"sme2d_l0", "sme2d_l1", "sme2d_l2", "sme2d_l4", "sme1d_l0_malpasset"} <= set(names)
    assert native.model_info("sme2d_l4")["n_dof_q"] == 12
    assert native.load().zsme_version().startswith(b"zsme")
