"""CPU: the C ABI library loads and exports every symbol include/*.h declares.

No compute call is made here; without a GPU, entry points must fail with a
status code (never crash) and say why.
"""
import ctypes as C
import glob
import os
import re

import pytest

import hnb200

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


# header -> the library that must export its symbols
HEADERS = {"hn_sm100.h": hnb200.LIB_PATH, "hn_host.h": hnb200.HOST_LIB_PATH}


def declared_symbols(header=None):
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        if header and os.path.basename(h) != header:
            continue
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"^\s*(?:const\s+)?\w+\**\s+\**(hn_\w+)\s*\(", text, flags=re.M))
    return sorted(names)


def test_every_header_has_a_library():
    assert {os.path.basename(h) for h in glob.glob(os.path.join(ROOT, "include", "*.h"))} <= set(HEADERS)


def test_header_declares_symbols():
    assert len(declared_symbols("hn_sm100.h")) >= 30 and len(declared_symbols("hn_host.h")) >= 10


def test_library_exports_every_declared_symbol():
    for header, path in HEADERS.items():
        lib = C.CDLL(path)
        missing = [s for s in declared_symbols(header) if not hasattr(lib, s)]
        assert not missing, (header, missing)


def test_binding_covers_every_declared_symbol():
    bound = set(hnb200.SIGNATURES) | set(hnb200.HOST_SIGNATURES)
    assert set(declared_symbols()) <= bound, set(declared_symbols()) - bound


def test_calls_before_init_fail_cleanly():
    lib = hnb200.load()
    st = lib.hn_spmv(None, 0, 1.0, None, 0.0, None, None)
    assert st == hnb200.HN_ERR_NOT_INITIALIZED or st == hnb200.HN_ERR_INVALID_ARG
    assert lib.hn_last_error()


def test_fault_injection_on_host():
    lib = hnb200.load()
    hnb200.fault_inject(0, hnb200.HN_ERR_INJECTED)
    assert lib.hn_csr_shape(None, None, None, None, None) == hnb200.HN_ERR_INJECTED
    assert b"injected" in lib.hn_last_error()
    # disarmed after firing: the next call reports its own error
    assert lib.hn_csr_shape(None, None, None, None, None) == hnb200.HN_ERR_INVALID_ARG


def test_missing_library_raises(tmp_path):
    hnb200_mod = hnb200
    saved = hnb200_mod._lib
    try:
        hnb200_mod._lib = None
        with pytest.raises(FileNotFoundError):
            hnb200_mod.load(str(tmp_path / "absent.so"))
    finally:
        hnb200_mod._lib = saved
