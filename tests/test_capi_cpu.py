"""The C ABI library without a GPU: it loads, exports every symbol that
include/*.h declares, and its host-only helpers behave (status strings, mask
sizes, the reference's test-mask generators).  No device computation here."""
import ctypes as C
import glob
import os
import re

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for hdr in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(hdr).read()
        names |= set(re.findall(r"DOL_API[^;(]*?\b(dol_\w+)\s*\(", text, flags=re.S))
    return sorted(names)


def test_library_exports_every_declared_symbol(dol):
    L = dol.lib()
    syms = declared_symbols()
    assert len(syms) > 30
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing


def test_status_strings_and_sizes(dol):
    L = dol.lib()
    assert L.dol_version() >= 1
    for code in range(6):
        assert L.dol_status_string(code)
    assert L.dol_mask_words(100, 100, 1) == 400
    assert L.dol_mask_words(32, 3, 2) == 6
    assert L.dol_mask_words(0, 3, 2) == 0
    assert L.dol_jumpflood_2d_workspace_size(10, 10) == 400
    assert L.dol_jumpflood_3d_workspace_size(4, 4, 4) == 2 * 512   # two 8-byte-cell buffers, 256-aligned


def test_host_generators_match_oracle(dol, O):
    for dims in [(64, 64), (100, 37), (1024, 1024)]:
        a = dol.add_points(np.zeros(dol.mask_words(*dims), np.uint32), dims, 100, 1)
        np.testing.assert_array_equal(a, O.add_points(O.new_mask(*dims), dims, 100, 1))
        for s in range(6):
            a = dol.add_block(np.zeros(dol.mask_words(*dims), np.uint32), dims, s)
            np.testing.assert_array_equal(a, O.add_block(O.new_mask(*dims), dims, s))
    for dims in [(16, 16, 16), (40, 33, 20)]:
        a = dol.add_points(np.zeros(dol.mask_words(*dims), np.uint32), dims, 50, 12345)
        np.testing.assert_array_equal(a, O.add_points(O.new_mask(*dims), dims, 50, 12345))
        for s in range(8):
            a = dol.add_block(np.zeros(dol.mask_words(*dims), np.uint32), dims, s)
            np.testing.assert_array_equal(a, O.add_block(O.new_mask(*dims), dims, s))


def test_calls_fail_cleanly_without_device_memory(dol):
    """A host pointer where device memory is required is rejected, not launched."""
    import torch
    if torch.cuda.is_available():
        buf = np.zeros(64, np.uint32)
        out = np.zeros(64 * 2, np.int16)
        st = dol.lib().dol_init_border_2d(C.c_int(32), C.c_int(2), buf.ctypes.data_as(C.c_void_p),
                                          out.ctypes.data_as(C.c_void_p), None)
        assert st == dol.ERR_INVALID_ARG
    else:
        st = dol.lib().dol_init_border_2d(C.c_int(32), C.c_int(2), None, None, None)
        assert st in (dol.ERR_CUDA, dol.ERR_INVALID_ARG)


def test_tuning_table_round_trip(dol):
    """dol_tune_set / dol_tune_get keep a value per family and width bucket
    (ceil(log2(w))), negative values included (DOL_TUNE_FASTSWEEP_3D: the
    anti-diagonal wavefront), and 0 restores the built-in heuristic."""
    L = dol.lib()
    FS3, OCC = 3, 11
    try:
        L.dol_tune_set(FS3, 256, -2)
        assert L.dol_tune_get(FS3, 256) == -2
        assert L.dol_tune_get(FS3, 200) == -2      # same bucket (129..256)
        assert L.dol_tune_get(FS3, 257) == 0       # next bucket untouched
        L.dol_tune_set(OCC, 1024, 1000)
        assert L.dol_tune_get(OCC, 1024) == 1000
        assert L.dol_tune_get(FS3, 256) == -2      # families are independent
    finally:
        L.dol_tune_set(FS3, 256, 0)
        L.dol_tune_set(OCC, 1024, 0)
    assert L.dol_tune_get(FS3, 256) == 0
