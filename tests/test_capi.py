"""The C-ABI library loads and exports every entry point include/*.h declares
(no compute calls: runs without a GPU)."""
import ctypes
import glob
import os
import re

import sipg

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        src = re.sub(r"//[^\n]*", "", src)
        for m in re.finditer(r"\b(sipg_[a-z0-9_]+)\s*\(", src):
            names.add(m.group(1))
    return names


def test_every_declared_symbol_is_exported():
    lib = sipg.lib()
    names = declared_functions()
    assert len(names) > 20
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_status_codes_and_errors_without_device():
    lib = sipg.lib()
    # invalid arguments are reported, never abort
    assert lib.sipg_ref_sizes(4, 1, None, None, None, None) == sipg.SIPG_INVALID_ARG
    assert b"dim" in lib.sipg_last_error()
    Np = ctypes.c_int()
    assert lib.sipg_ref_sizes(3, 3, ctypes.byref(Np), None, None, None) == sipg.SIPG_OK
    assert Np.value == 20
    assert lib.sipg_op_create(None, 3, 1, None) == sipg.SIPG_INVALID_ARG


def test_host_mesh_build_needs_no_device():
    mesh = sipg.Mesh.box(3, 2, jitter=0.1, seed=3)
    e = mesh.export(3)
    assert e["K"] == 48 and e["Kb"] == 48
