"""The C-ABI library loads and exports every entry point include/magasm.h declares.

CPU only: loading libmagasm.so makes no CUDA call, so this runs without a GPU.
"""
import ctypes
import os
import re

from conftest import ROOT

from magpackage_b200 import _lib

HEADER_DIR = os.path.join(ROOT, "include")


def declared_symbols():
    names = set()
    for fn in os.listdir(HEADER_DIR):
        if not fn.endswith(".h"):
            continue
        text = open(os.path.join(HEADER_DIR, fn)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(mag_\w+)\s*\(", text, re.M):
            names.add(m.group(1))
    return names


def test_library_built_for_sm100a():
    assert os.path.exists(_lib.LIB_PATH), "build libmagasm.so first (magpackage_b200/build.py)"


def test_every_declared_symbol_is_exported():
    lib = ctypes.CDLL(_lib.LIB_PATH)
    names = declared_symbols()
    assert len(names) >= 15
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header():
    assert set(_lib.exported_symbols()) == declared_symbols()


def test_version_and_error_text_without_gpu():
    lib = _lib.load()
    assert lib.mag_version() >= 1
    assert isinstance(lib.mag_last_error(), bytes)
    # argument validation happens before any CUDA call
    rc = lib.mag_mesh_get_info(None, None)
    assert rc == -1 and b"bad arguments" in lib.mag_last_error()


def test_mex_entry_points_accept_an_empty_mesh():
    """The reference gateways return empty triplets for zero elements; so do these, without
    touching the GPU (so this runs on the CPU)."""
    L = _lib.load()
    p = (ctypes.c_double * 4)()
    args_j = [p, 1, p, 0, p, p, p, p, 1, p, 4, p, p, p, p, 1, p, 1, p, 4, p, p, p, 1, p, p, p, p, p]
    assert L.mag_mex_jacobian(*args_j) == 0
    assert L.mag_mex_curl_curl(p, 1, p, 0, p, p, p, p, 4, p, p, p, p) == 0
    assert L.mag_mex_mass(p, 1, p, 0, p, p, None, 0, p, 4, p, p, p, p) == 0


def test_product_path_fails_loudly_without_its_library_or_a_gpu(monkeypatch):
    """No CPU fallback: a missing library and a machine without a CUDA device are errors."""
    import pytest
    import torch

    monkeypatch.setattr(_lib, "_LIB", None)
    with pytest.raises(FileNotFoundError):
        _lib.load(os.path.join(ROOT, "no_such_dir", "libmagasm.so"))
    monkeypatch.setattr(torch.cuda, "is_available", lambda: False)
    with pytest.raises(RuntimeError, match="no CPU path"):
        _lib.lib()
