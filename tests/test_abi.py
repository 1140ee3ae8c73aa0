"""The C-ABI library loads on a CPU-only host and exports every entry point
declared in include/fvmhd3d_b200.h; without a GPU it fails loudly."""
import ctypes
import os
import re

import pytest

from common import ROOT

HEADER = os.path.join(ROOT, "include", "fvmhd3d_b200.h")


def declared():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(fvm_[a-z0-9_]+)\s*\(", src)))


def test_header_lists_entry_points():
    names = declared()
    assert "fvm_step" in names and "fvm_slope_limiter" in names and len(names) >= 20


def test_library_exports_every_declared_symbol():
    from fvmhd3d_b200 import _lib
    so = _lib.lib()
    for name in declared():
        assert hasattr(so, name), name
        assert name in _lib.SIGNATURES, name


def test_fails_loudly_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import fvmhd3d_b200 as F
    with pytest.raises(F.FvmError):
        F.System()


def test_missing_library_raises(monkeypatch, tmp_path):
    from fvmhd3d_b200 import _lib
    monkeypatch.setattr(_lib, "_LIB", None)
    monkeypatch.setattr(_lib, "SO_PATH", str(tmp_path / "absent.so"))
    with pytest.raises(RuntimeError):
        _lib.lib()
