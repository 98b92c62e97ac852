"""The no-allocation equalize entry point against the scratch-taking one.

mb_equalize_tc_noalloc serves callers that cannot call cudaMalloc when they
equalize (real-time threads kept out of the driver's allocator, or memory
fixed at start-up by a framework that owns all allocations): its scratch is a
fixed array inside the library.  Its results must equal those of
mb_equalize_tc (the same kernels, so the comparison is exact, which is within
the 1% / |LLR| > 4 tolerance of the tensor-core tests), on two calls in a row,
the second reusing the scratch the first one left behind.  This file sorts
last so that a stop-at-first-failure run has executed every other test first.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _p(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _run(L, fn, W, y, K, M, S, sg, n_sym, Qm, cb, stride, zeros, scr, scratch):
    llr = torch.zeros(n_sym, K, stride, dtype=torch.float16, device="cuda")
    n_valid = min(S * Qm, cb)
    hard = torch.zeros(n_sym, K, (n_valid + 7) // 8, dtype=torch.uint8, device="cuda")
    x = torch.zeros(n_sym, K, S, dtype=torch.complex64, device="cuda")
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    args = [_p(W), _p(y), K, M, S, sg, n_sym, Qm, cb, stride, zeros, 1, _p(llr), _p(hard), scr, _p(x)]
    if scratch is not None:
        args += [_p(scratch[0]), _p(scratch[1])]
    status = fn(*args, stream)
    torch.cuda.synchronize()
    return status, llr.cpu().numpy().view(np.uint16), hard.cpu().numpy(), x.cpu().numpy()


@pytest.mark.parametrize("K,M,S,sg,n_sym,Qm", [(32, 256, 3276, 16, 12, 6), (16, 64, 1200, 16, 3, 4)])
def test_noalloc_matches_scratch_entry_point_twice(K, M, S, sg, n_sym, Qm):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from megastation_b200 import _lib
    from megastation_b200.ops import Scrambler
    L = _lib.LIB
    rng = np.random.default_rng(K + n_sym)
    G = (S + sg - 1) // sg
    cb, zeros = (S * Qm * 9) // 10 // Qm * Qm, 2 * Qm
    stride = cb + zeros + 4
    scr = Scrambler()
    img, ylp = _lib.U64(), _lib.U64()
    assert L.mb_equalize_tc_scratch(K, M, S, sg, n_sym, ctypes.byref(img), ctypes.byref(ylp)) == 0
    scratch = (torch.empty(img.value, dtype=torch.uint8, device="cuda"),
               torch.empty(ylp.value, dtype=torch.uint8, device="cuda"))
    for call in range(2):
        # different inputs per call: the second call must not see the first
        W = _dev(((rng.standard_normal((G, M, K)) + 1j * rng.standard_normal((G, M, K)))
                  / np.sqrt(2 * M)).astype(np.complex64))
        y = _dev(((rng.standard_normal((n_sym, M, S)) + 1j * rng.standard_normal((n_sym, M, S)))
                  / np.sqrt(2)).astype(np.complex64))
        st_ref, llr_ref, hard_ref, x_ref = _run(L, L.mb_equalize_tc, W, y, K, M, S, sg, n_sym, Qm, cb,
                                                stride, zeros, scr._h, scratch)
        st_na, llr_na, hard_na, x_na = _run(L, L.mb_equalize_tc_noalloc, W, y, K, M, S, sg, n_sym, Qm,
                                            cb, stride, zeros, scr._h, None)
        assert st_ref == 0 and st_na == 0, (call, st_ref, st_na)
        np.testing.assert_array_equal(llr_na, llr_ref)
        np.testing.assert_array_equal(hard_na, hard_ref)
        np.testing.assert_array_equal(x_na, x_ref)
        assert np.abs(x_ref).max() > 0


def test_noalloc_rejects_oversized_request():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from megastation_b200 import _lib
    L = _lib.LIB
    # 1024 antennas x 64 users x 8192 subcarriers: the detector images alone
    # exceed the fixed scratch; the entry point must refuse before any launch
    K, M, S, sg, Qm = 64, 1024, 8192, 16, 2
    dummy = torch.zeros(16, dtype=torch.uint8, device="cuda")
    p = ctypes.c_void_p(dummy.data_ptr())
    cb = S * Qm
    status = L.mb_equalize_tc_noalloc(p, p, K, M, S, sg, 1, Qm, cb, cb, 0, 1, p, None, None, None, None)
    assert status == _lib.MB_TOO_LARGE
    assert "scratch" in _lib.status_str(status)
