"""The C ABI: the library loads, exports every entry point include/prtlb.h
declares, and its struct layouts match the ctypes mirrors.  No GPU needed."""

import ctypes
import os
import re

from conftest import ROOT

from prtlb_gpu import _lib

HEADER = os.path.join(ROOT, "include", "prtlb.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(prt_[a-z0-9_]+)\s*\(", text)))


def test_every_declared_symbol_is_exported_and_bound():
    L = _lib.lib()
    names = declared_functions()
    assert "prt_flow" in names and "prt_adr_run" in names
    for n in names:
        assert hasattr(L, n), n
        assert n in _lib._PROTOS, "no ctypes prototype for %s" % n


def test_struct_layouts_match():
    L = _lib.lib()
    for i, cls in enumerate(_lib.SIZEOF_ORDER):
        assert L.prt_sizeof(i) == ctypes.sizeof(cls), cls.__name__
    assert L.prt_sizeof(99) == 0
    assert L.prt_abi_version() == 1


def test_null_arguments_are_refused_without_a_device():
    L = _lib.lib()
    assert L.prt_create(0, None) == _lib.PRT_E_INVALID
    assert L.prt_flow(None, None, None, None, None) == _lib.PRT_E_INVALID
    assert L.prt_adr_run(None, None, _lib.PROGRESS_CB(), None, None) == _lib.PRT_E_INVALID
