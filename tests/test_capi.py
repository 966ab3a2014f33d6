"""The C-ABI library loads and exports every function include/tictac_b200.h declares."""
import ctypes
import os
import re

import tictac_b200 as tt
from conftest import ROOT


def declared_functions():
    src = open(os.path.join(ROOT, "include", "tictac_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(tt_[A-Za-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    lib = tt.load()
    names = declared_functions()
    assert len(names) >= 30
    for name in names:
        assert hasattr(lib, name), f"{name} declared in include/tictac_b200.h but not exported"
    assert set(names) == set(tt.EXPORTED_SYMBOLS)


def test_error_paths_without_device():
    lib = tt.load()
    run = ctypes.c_void_p()
    bad = (ctypes.c_char_p * 1)(b"Np_WP")
    assert lib.tt_run_create(ctypes.byref(run), 1, bad) == tt.TT_ERR_BADARG
    assert b"=" in lib.tt_last_error_string()
    assert lib.tt_run_num_channels(None, None) == tt.TT_ERR_BADARG
    rp = tt.run_params()
    assert rp.Nphi == 48 and rp.Nx == 48 and rp.precision == tt.PRECISION_MIXED
