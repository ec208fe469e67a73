"""C ABI checks that need no GPU: the library builds, loads and exports
every function include/mzk.h declares; context creation fails cleanly when no
device is present."""
import re

import pytest

from _loader import load

mzk = load()


def header_functions():
    text = mzk.HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(mzk_\w+)\s*\(", text)))


def test_library_exports_every_header_symbol():
    lib = mzk.lib()
    names = header_functions()
    assert len(names) >= 15
    for name in names:
        assert hasattr(lib, name), name
        assert name in mzk.SIGNATURES, f"{name} lacks a ctypes signature"
    assert set(mzk.SIGNATURES) == set(names)


def test_version_string():
    assert b"sm_100a" in mzk.lib().mzk_version()


def test_pick_window_is_monotone():
    cs = [mzk.msm_pick_window(1 << k) for k in range(4, 27)]
    assert all(5 <= c <= 24 for c in cs)
    assert cs == sorted(cs)


def test_context_without_device_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(mzk.MzkError):
        mzk.Context(0)
