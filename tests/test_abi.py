"""The C-ABI library loads on a machine without a GPU and exports every declared entry point."""
import ctypes as C
import os
import re

import pytest

from cleo_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    txt = open(os.path.join(ROOT, "include", "cleo_b200.h")).read()
    return sorted(set(re.findall(r"\b(cleo_b200_[a-z_0-9]+)\s*\(", txt)))


def test_header_declares_abi():
    names = declared_functions()
    assert set(abi.EXPORTED) <= set(names), set(abi.EXPORTED) - set(names)
    assert set(names) <= set(abi.EXPORTED), set(names) - set(abi.EXPORTED)


@pytest.mark.skipif(not abi.LIB_PATH.exists(), reason="library not built")
def test_library_exports_every_symbol():
    lib = C.CDLL(str(abi.LIB_PATH))
    for name in declared_functions():
        assert hasattr(lib, name), name
    lib.cleo_b200_version.restype = C.c_char_p
    assert b"sm_100a" in lib.cleo_b200_version()


def test_struct_sizes_match_header_layout():
    # cleo_b200_params: 4 u32 + 4 f64 + (i32,u32) + 2 f64 + 2 i32 + 2 f64 + 2 i32 + f64
    #                   + 2 i32 + f64 + u64 + 2 i32 + 2 i32
    assert C.sizeof(abi.Params) == 16 + 32 + 8 + 16 + 8 + 16 + 8 + 8 + 8 + 8 + 8 + 8 + 8
    assert C.sizeof(abi.Grid) == 4 + 12 + 13 * 8
    assert C.sizeof(abi.Supers) == 8 * 8
    assert C.sizeof(abi.GbxState) == 11 * 8
    assert C.sizeof(abi.Error) == 16


def test_missing_library_fails_loudly(tmp_path):
    with pytest.raises(FileNotFoundError):
        abi.load_library(tmp_path / "nope.so")
