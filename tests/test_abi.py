"""The C-ABI library builds, loads and exports every symbol of include/cufhe_b200.h
(no compute calls: these run without a GPU)."""
import ctypes as C
import re
from pathlib import Path

import pytest

from cufhepp_b200 import engine

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    text = (ROOT / "include" / "cufhe_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(cufhe_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_gate_api():
    names = declared_functions()
    for must in ["cufhe_initialize", "cufhe_cleanup", "cufhe_synchronize", "cufhe_gate",
                 "cufhe_gate_batch", "cufhe_stream_create", "cufhe_stream_query"]:
        assert must in names


def test_library_exports_every_declared_symbol():
    lib = engine.load()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header():
    assert set(declared_functions()) == set(engine.SIGNATURES)


def test_errors_without_initialize():
    lib = engine.load()
    # argument checks happen before any device work
    assert lib.cufhe_set_precision(7) == -1
    assert b"precision" in lib.cufhe_last_error()
    assert lib.cufhe_initialize(None) == -1
    kv = engine.KeyView(0, 0, 0, 0, 0)
    assert lib.cufhe_initialize(C.byref(kv)) == -1


def test_wrong_key_sizes_rejected():
    import numpy as np
    lib = engine.load()
    bk = np.zeros(10, np.uint32)
    ksk = np.zeros(10, np.uint32)
    kv = engine.KeyView(bk.ctypes.data, bk.size, ksk.ctypes.data, ksk.size, 1)
    assert lib.cufhe_initialize(C.byref(kv)) == -1
    assert b"words" in lib.cufhe_last_error()


def test_gate_before_initialize_is_state_error():
    import numpy as np
    lib = engine.load()
    x = np.zeros(1025, np.uint32)
    rc = lib.cufhe_gate(0, 1, x.ctypes.data_as(C.c_void_p), x.ctypes.data_as(C.c_void_p),
                        x.ctypes.data_as(C.c_void_p), None, None)
    assert rc in (-2, -3)  # not initialized (or no device at all)


def test_bad_gate_id_rejected():
    lib = engine.load()
    assert lib.cufhe_gate(99, 1, None, None, None, None, None) == -1


def test_lvl02_entry_points_check_state_and_sizes():
    import numpy as np
    lib = engine.load()
    assert lib.cufhe_initialize_lvl02(None) == -1
    bk = np.zeros(10, np.uint64)
    ksk = np.zeros(10, np.uint32)
    kv = engine.KeyView(bk.ctypes.data, bk.size, ksk.ctypes.data, ksk.size, 1)
    assert lib.cufhe_initialize_lvl02(C.byref(kv)) == -1
    assert b"lvl02 bootstrapping key" in lib.cufhe_last_error()
    x = np.zeros(2049, np.uint64)
    p = x.ctypes.data_as(C.c_void_p)
    # lvl02 gates and path pieces refuse to run before cufhe_initialize_lvl02
    assert lib.cufhe_gate(0, 2, p, p, p, None, None) in (-2, -3)
    assert lib.cufhe_blind_rotate_lvl02(p, 1, 1 << 61, -1, p, None, None) == -2
    assert b"initialize_lvl02" in lib.cufhe_last_error()
    assert lib.cufhe_identity_keyswitch_lvl20(p, 1, p, None) == -2
    assert lib.cufhe_gate(0, 3, p, p, p, None, None) == -1  # no level 3
