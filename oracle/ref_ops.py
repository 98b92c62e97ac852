"""ctypes loader for oracle/_ref/libref_ops.so: the reference's own CUDA
operators (cuFFT FFTs, cuBLAS/cuSOLVER beamformer, SIMT equalizer) built
from the reference tree by oracle/ref_ops.mk.

TEST INFRASTRUCTURE ONLY: used by tests/ as a parity check against the
reference implementation itself and by bench.py's reference arm; the product
package never loads it.  available() is False where the library was not
built (no reference tree at build time).
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
PATH = os.path.join(_HERE, "_ref", "libref_ops.so")
_LIB = None


def available():
    return os.path.exists(PATH)


def lib():
    global _LIB
    if _LIB is None:
        L = ctypes.CDLL(PATH)
        VP, U32, U64 = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64
        L.ref_slot_create.restype = VP
        L.ref_slot_create.argtypes = [U32] * 8 + [U64] * 3
        L.ref_slot_create_iq.restype = VP
        L.ref_slot_create_iq.argtypes = [U32] * 8 + [U64] * 3 + [U32]
        L.ref_slot_destroy.argtypes = [VP]
        L.ref_slot_uplink.restype = ctypes.c_int
        L.ref_slot_uplink.argtypes = [VP, VP, VP, VP]
        L.ref_slot_csi.restype = VP
        L.ref_slot_csi.argtypes = [VP]
        _LIB = L
    return _LIB


class RefSlot:
    """One cell's uplink slot through the reference operators: int16 IQ, or
    int8 IQ (the reference's production sample type) with iq="int8"."""

    def __init__(self, M, K, N, S, sg, Qm, P, U, cb_size, zeros, cb_stride, iq="int16"):
        if iq not in ("int16", "int8"):
            raise ValueError("the reference FFT takes int16 or int8 samples")
        self._h = lib().ref_slot_create_iq(M, K, N, S, sg, Qm, P, U, cb_size, zeros, cb_stride,
                                           1 if iq == "int8" else 0)
        if not self._h:
            raise RuntimeError("ref_slot_create failed")

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _LIB is not None:
            _LIB.ref_slot_destroy(h)
            self._h = None

    def uplink(self, iq_ptr, llr_ptr, stream_ptr):
        rc = lib().ref_slot_uplink(self._h, iq_ptr, llr_ptr, stream_ptr)
        if rc:
            raise RuntimeError(f"ref_slot_uplink failed ({rc})")

    def csi_ptr(self):
        return lib().ref_slot_csi(self._h)
