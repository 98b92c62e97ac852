"""The bounded device wait gives up with an error the host reads.

Every mbarrier wait of the tensor-core kernels is bounded by wall time and,
when it runs out, ORs the timeout bit into the device error word instead of
spinning forever.  mb_selftest_wait runs that same wait on a barrier that
nothing arrives on (arm = 0), with a short limit, so the wait must run out:
the kernel returns, the context stays usable, and mb_device_error reports
bit 1.  With the barrier armed the wait completes and no bit is set."""
import ctypes

import pytest
import torch

pytestmark = pytest.mark.gpu


def test_expired_wait_reports_timeout_and_context_survives():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from megastation_b200 import _lib, ops
    L = _lib.LIB
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    ops.device_error(clear=True)
    # armed barrier: completes, no error bit
    assert L.mb_selftest_wait(1_000_000, 1, stream) == _lib.MB_OK
    assert ops.device_error(clear=True) == 0
    # a barrier nothing arrives on: the 2 ms limit runs out, bit 1 is set
    assert L.mb_selftest_wait(2_000_000, 0, stream) == _lib.MB_OK
    assert ops.device_error(clear=True) & 1 == 1
    # cleared, and the context still runs work
    assert ops.device_error(clear=True) == 0
    x = torch.arange(1024, device="cuda", dtype=torch.float32)
    assert float(x.sum()) == 1024 * 1023 / 2
    # limits outside (0, 1 s] are refused on the host
    assert L.mb_selftest_wait(0, 0, stream) == _lib.MB_BAD_ARG
    assert L.mb_selftest_wait(2_000_000_000, 0, stream) == _lib.MB_BAD_ARG
