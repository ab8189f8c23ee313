"""The C-ABI library: loads on any machine and exports what the header declares."""
import ctypes as C
import os
import re

import pytest

from conftest import ROOT

from parallelcmacionize_b200 import _lib

HEADER = os.path.join(ROOT, "include", "cmacionize_b200.h")


def declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|void|const char \*)\s*(cmi_\w+)\s*\(", text,
                                 re.MULTILINE)))


def test_header_declares_the_binding_list():
    assert declared_functions() == sorted(_lib.EXPORTED)


def test_library_exports_every_declared_symbol():
    L = _lib.load()
    for name in declared_functions():
        assert hasattr(L, name), name
    assert L.cmi_abi_version() == 2  # 2: cmi_stats.packets_reemitted


def test_default_options():
    o = _lib.default_options()
    assert o.transport_precision == _lib.TRANSPORT_MIXED
    assert o.balance_form == _lib.BALANCE_STABLE
    assert o.tally_mode == _lib.TALLY_FIXED64 and o.use_graph == 1
    with pytest.raises(TypeError):
        _lib.default_options(no_such_option=1)


def test_struct_layouts_match_header():
    assert C.sizeof(_lib.GridDesc) == 6 * 8 + 6 * 4 + 2 * 8
    assert C.sizeof(_lib.Options) == 16 * 4
    assert C.sizeof(_lib.Stats) == 6 * 8 + 2 * 4 + 8
    assert _lib.PHOTON_DTYPE.itemsize == 80
    assert C.sizeof(_lib.DustStats) == 7 * 8 + 2 * 4


def test_null_arguments_fail_cleanly():
    L = _lib.load()
    assert L.cmi_create(None, 1, None, None) == _lib.ERR_INVALID_ARGUMENT
    assert L.cmi_synchronize(None) == _lib.ERR_INVALID_ARGUMENT
    assert b"null" in L.cmi_last_error_string()
    assert L.cmi_destroy(None) == _lib.OK
    assert L.cmi_dust_run(None, 0, 10, 1, 0, 0.5, None, 4, 4, None, None) == \
        _lib.ERR_INVALID_ARGUMENT
    assert L.cmi_walk_photons(None, 0, 0, 1, None, None, 1, None) == _lib.ERR_INVALID_ARGUMENT
