"""CPU-side checks of the C ABI: the library loads, exports every entry point
include/ldpc_b200.h declares, and its host-only paths (codes, schedules,
argument validation) behave; no GPU call is made here."""
import ctypes
import os
import re

import numpy as np
import pytest

import fast_ldpc_decoder_for_gpu_fixed_b200 as fl
from fast_ldpc_decoder_for_gpu_fixed_b200 import _lib
from fast_ldpc_decoder_for_gpu_fixed_b200.decoder import NativeCode

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "ldpc_b200.h")


def declared():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", " ", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(ldpc_[a-z0-9_]+)\s*\(", txt)))


def test_header_symbols_exported():
    L = _lib.lib()
    names = declared()
    assert len(names) >= 14
    for name in names:
        assert hasattr(L, name), name
    assert set(names) == set(_lib.SIGNATURES), "python binding out of sync with the header"


def test_header_constants_match_python():
    """Every status code, kind, packing, flag and output format the header defines has
    the same value in the Python binding."""
    txt = open(HEADER).read()
    defs = {k: int(v) for k, v in re.findall(r"#define\s+(LDPC_[A-Z0-9_]+)\s+\(?(-?\d+)\)?", txt)}
    expect = {"LDPC_OK": _lib.LDPC_OK, "LDPC_OUT_BYTES": _lib.OUT_BYTES, "LDPC_OUT_PACKED": _lib.OUT_PACKED,
              "LDPC_FLAG_EARLY_STOP": _lib.FLAG_EARLY_STOP,
              "LDPC_FLAG_EARLY_STOP_FRAMES": _lib.FLAG_EARLY_STOP_FRAMES,
              "LDPC_BATCH_GRAPH": _lib.BATCH_GRAPH,
              "LDPC_EARLY_STOP_DEFAULT_SLACK": _lib.EARLY_STOP_DEFAULT_SLACK,
              "LDPC_EARLY_SLACK_ANY": _lib.EARLY_SLACK_ANY,
              "LDPC_TRAIN_QUANTIZED": _lib.TRAIN_QUANTIZED, "LDPC_TRAIN_FRAME_LOSS": _lib.TRAIN_FRAME_LOSS}
    expect.update({v: k for k, v in _lib.ERRORS.items()})
    expect.update({"LDPC_" + k: v for k, v in _lib.KINDS.items() if k != "FMS"})
    expect.update({"LDPC_PACK_" + k: v for k, v in _lib.PACKS.items()})
    for name, value in expect.items():
        assert defs.get(name) == value, (name, defs.get(name), value)
    # the flags are distinct bits
    flags = [defs["LDPC_FLAG_EARLY_STOP"], defs["LDPC_FLAG_EARLY_STOP_FRAMES"], defs["LDPC_BATCH_GRAPH"]]
    assert all(f & (f - 1) == 0 for f in flags) and len(set(flags)) == 3


def test_version_and_error_string():
    assert _lib.lib().ldpc_version() >= 1
    assert isinstance(_lib.last_error(), str)


@pytest.mark.parametrize("name", fl.reference_tables())
def test_code_objects_and_schedule(name):
    code = fl.load_table(name)
    info = NativeCode(code).info()
    assert (info["n"], info["checks"], info["edges"]) == (code.n, code.m, code.e)
    assert info["dmax"] == int(code.degrees.max())
    assert info["n_info"] == code.n - code.m


def test_schedule_levels_restated():
    """The level counts the library reports equal an independent restatement."""
    for name in ("4000x2000", "576x288", "1944x972", "2048x384"):
        code = fl.load_table(name)
        last = np.full(code.n, -1)
        lev = []
        for r in code.rows():
            L = int(last[r].max()) + 1
            lev.append(L)
            last[r] = L
        info = NativeCode(code).info()
        assert info["levels"] == max(lev) + 1
        assert info["widest_level"] == int(np.bincount(lev).max())
        # rows of a level never share a variable
        lev = np.array(lev)
        for L in range(max(lev) + 1):
            vs = np.concatenate([code.cols[code.row_ptr[r]:code.row_ptr[r + 1]] for r in np.flatnonzero(lev == L)])
            assert len(vs) == len(set(vs.tolist()))


def test_create_from_table_matches_csr():
    code = fl.load_table("576x288")
    h = ctypes.c_void_p()
    pos = code.cols.astype(np.uint32)
    _lib.check(_lib.lib().ldpc_code_create_from_table(ctypes.byref(h), 576, 288, 1824, 2, 7, 96, 6, 192,
                                                      pos.ctypes.data))
    a = (ctypes.c_int * 8)()
    _lib.check(_lib.lib().ldpc_code_info(h, a))
    _lib.lib().ldpc_code_destroy(h)
    assert list(a)[:7] == list(NativeCode(code).info().values())


def test_code_load_file():
    h = ctypes.c_void_p()
    path = os.path.join(os.path.dirname(fl.codes.__file__), "codes", "4000x2000.ldpc")
    _lib.check(_lib.lib().ldpc_code_load(ctypes.byref(h), path.encode()))
    a = (ctypes.c_int * 8)()
    _lib.check(_lib.lib().ldpc_code_info(h, a))
    _lib.lib().ldpc_code_destroy(h)
    assert list(a)[:4] == [4000, 2000, 12000, 6]


def test_bad_codes_rejected():
    L = _lib.lib()
    h = ctypes.c_void_p()
    rp = np.array([0, 3, 6], dtype=np.int32)
    cols = np.array([0, 1, 2, 1, 2, 9], dtype=np.int32)  # 9 >= n
    assert L.ldpc_code_create(ctypes.byref(h), 5, 2, rp.ctypes.data, cols.ctypes.data, None) == -1
    assert "outside" in _lib.last_error()
    cols[5] = 3
    rp_bad = np.array([0, 3, 3], dtype=np.int32)  # empty row
    assert L.ldpc_code_create(ctypes.byref(h), 5, 2, rp_bad.ctypes.data, cols.ctypes.data, None) == -1
    assert L.ldpc_code_create(None, 5, 2, rp.ctypes.data, cols.ctypes.data, None) == -1
    assert L.ldpc_code_create(ctypes.byref(h), 70000, 2, rp.ctypes.data, cols.ctypes.data, None) == -3
    pos = np.zeros(10, dtype=np.uint32)
    assert L.ldpc_code_create_from_table(ctypes.byref(h), 10, 2, 10, 1, 6, 2, 0, 0, pos.ctypes.data) == -1
    assert L.ldpc_code_load(ctypes.byref(h), b"/nonexistent.ldpc") == -1
    assert L.ldpc_decode_host(None, None, None, 20) == -1
