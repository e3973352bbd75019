"""The C-ABI library builds, loads and exports every entry point include/efs.h declares.

No compute call is made, so this runs without a GPU.
"""
import ctypes
import os
import re
import subprocess

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "efs.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(efs_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ("efs_create", "efs_init", "efs_iterate", "efs_configure_pml", "efs_configure_mur",
                 "efs_configure_nf2ff", "efs_far_field", "efs_energy", "efs_get_fields", "efs_destroy"):
        assert must in names


def test_library_exports_every_declared_symbol():
    from efs_b200.build import build
    lib_path = build()
    lib = ctypes.CDLL(lib_path)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", lib_path], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (efs_[a-z0-9_]+)", out))
    assert set(declared_functions()) <= exported


def test_python_binding_covers_header():
    from efs_b200 import _lib
    assert set(declared_functions()) == set(_lib.SIGNATURES)


def test_create_without_device_fails_cleanly():
    """efs_create returns an error code (never aborts) when no device is usable."""
    import torch
    if torch.cuda.is_available():
        return
    from efs_b200 import _lib
    lib = _lib.load()
    h = ctypes.c_void_p()
    rc = lib.efs_create(ctypes.byref(h), 0)
    assert rc == 3 and not h.value
    assert lib.efs_last_error(None)
