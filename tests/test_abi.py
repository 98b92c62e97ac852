"""CPU-side checks of the C ABI: the library loads, exports every function
include/megastation_b200.h declares, and validates arguments on the host
before touching a device."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            text = open(os.path.join(ROOT, "include", fn)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names |= set(re.findall(r"\b(mb_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_functions()
    for n in ["mb_fft_uplink", "mb_fft_pilot", "mb_ifft_downlink", "mb_zf_uplink", "mb_zf_precoder",
              "mb_equalize", "mb_precode", "mb_modulate", "mb_scramble"]:
        assert n in names


def test_library_exports_every_declared_symbol():
    from megastation_b200 import _lib
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_status_strings_and_version():
    from megastation_b200 import _lib
    assert _lib.status_str(0) == "ok"
    assert "shape" in _lib.status_str(1)
    assert b"sm_100a" in _lib.LIB.mb_version()


def test_host_tables_match_oracle():
    import megastation_b200 as mb
    from oracle import oracle as orc
    for S in (16, 600, 1200, 3276):
        np.testing.assert_allclose(mb.pilot_sign(S).numpy(), orc.pilot_sign(S), atol=1e-6)
    for S, Qm in [(1200, 4), (3276, 6), (600, 2), (3276, 8)]:
        assert mb.ldpc_sizes(S, Qm) == orc.ldpc_sizes(S, Qm)
        assert mb.ldpc_sizes(S, Qm, downlink=True, pilot_spacing=16) == \
            orc.ldpc_sizes(S, Qm, downlink=True, pilot_spacing=16)


def test_host_validation_rejects_bad_shapes():
    from megastation_b200 import _lib
    L = _lib.LIB
    h = ctypes.c_void_p()
    d = _lib.MbFftDesc(0, 3000, 1200, 64, 16, 16)  # N not a power of two
    assert L.mb_fft_create(ctypes.byref(d), ctypes.byref(h)) == _lib.MB_BAD_SHAPE
    d = _lib.MbFftDesc(0, 2048, 4096, 64, 16, 16)  # S > N
    assert L.mb_fft_create(ctypes.byref(d), ctypes.byref(h)) == _lib.MB_BAD_SHAPE
    assert L.mb_zf_create(8, 16, 10, ctypes.byref(h)) == _lib.MB_BAD_SHAPE  # K > M
    assert L.mb_zf_create(256, 65, 10, ctypes.byref(h)) == _lib.MB_BAD_SHAPE  # K > 64
    assert L.mb_fft_uplink(None, None, 0, 1, None, None) == _lib.MB_BAD_ARG
    assert L.mb_equalize(None, None, 4, 8, 16, 16, 1, 2, 32, 32, 0, 1, None, None, None, None, None) \
        == _lib.MB_BAD_ARG
    # bad modulation order / cb layout are rejected before any launch
    p = ctypes.c_void_p(16)
    assert L.mb_equalize(p, p, 4, 8, 16, 16, 1, 3, 32, 32, 0, 1, p, None, None, None, None) == _lib.MB_BAD_ARG
    assert L.mb_equalize(p, p, 4, 8, 16, 16, 1, 2, 32, 16, 0, 1, p, None, None, None, None) == _lib.MB_BAD_SHAPE
    assert L.mb_modulate(p, p, 4, 16, 1, 5, 0, None, None) == _lib.MB_BAD_ARG
