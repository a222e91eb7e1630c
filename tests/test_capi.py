"""The C-ABI library loads and exports every entry point include/fresco_b200.h declares (no GPU calls)."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "fresco_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(fresco_[A-Za-z0-9_]+)\s*\(", src)))


def test_header_symbols_exported():
    from fresco_b200 import _lib

    lib = ctypes.CDLL(_lib.LIB_PATH)
    names = declared_symbols()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header():
    from fresco_b200 import _lib

    assert sorted(_lib.exported_symbols()) == declared_symbols()


def test_abi_version_and_error_string():
    from fresco_b200 import _lib

    assert _lib.lib.fresco_abi_version() == 100
    assert isinstance(_lib.lib.fresco_last_error(), bytes)


def test_argument_errors_before_device_work():
    """Shape errors raise the reference's exception types without touching the GPU."""
    import numpy as np
    import pytest

    from fresco_b200 import NUwU

    with pytest.raises(AssertionError):  # nuwu.pyx:17
        NUwU(np.ones(4), 2, np.zeros(25), np.ones(24), np.ones(2))
    with pytest.raises(ValueError):
        NUwU(np.ones(4), 2, np.zeros(25), np.ones(25), np.ones(2), precision="fp16")
