"""ctypes loader for the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() and
by the CPU-baseline leg of bench.py, as the checker.  The product package
(megastation_b200) never imports it.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

F32P = ctypes.POINTER(ctypes.c_float)
U16P = ctypes.POINTER(ctypes.c_uint16)
U8P = ctypes.POINTER(ctypes.c_uint8)
F64P = ctypes.POINTER(ctypes.c_double)
U64 = ctypes.c_uint64
U32 = ctypes.c_uint32
VP = ctypes.c_void_p


def build():
    subprocess.check_call(["make", "-s", "-C", _HERE])


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        _LIB = ctypes.CDLL(path)
        L = _LIB
        L.orc_f2h.restype = ctypes.c_uint16
        L.orc_f2h.argtypes = [ctypes.c_float]
        L.orc_h2f.restype = ctypes.c_float
        L.orc_h2f.argtypes = [ctypes.c_uint16]
        L.orc_zadoff_chu.argtypes = [U64, F32P]
        L.orc_cyclic_shift.argtypes = [F32P, F32P, U64, ctypes.c_float]
        L.orc_pilot_sign.argtypes = [U64, F32P]
        L.orc_dmrs_table.argtypes = [U64, U64, F32P]
        L.orc_scrambler_seq127.argtypes = [U8P]
        L.orc_scramble_bytes.argtypes = [U8P, U8P, U64, U64]
        L.orc_gold_seq.argtypes = [U32, U64, U8P]
        L.orc_mod_table.argtypes = [ctypes.c_int, F32P]
        L.orc_modulate.argtypes = [U8P, F32P, U64, U64, U64, ctypes.c_int, U32, F32P]
        L.orc_demod.argtypes = [ctypes.c_int, ctypes.c_float, ctypes.c_float, U16P]
        L.orc_fft_d.argtypes = [F64P, U32, ctypes.c_int]
        L.orc_uplink_fft.argtypes = [VP, ctypes.c_int, U32, U32, U32, U32, F32P]
        L.orc_pilot_fft.argtypes = [VP, ctypes.c_int, U32, U32, U32, U32, U32, U32, U32, F32P, F32P]
        L.orc_ifft_downlink.argtypes = [F32P, U32, U32, ctypes.c_int, VP]
        L.orc_zf.restype = ctypes.c_int
        L.orc_zf.argtypes = [F32P, U32, U32, U32, U32, U32, F32P, F64P]
        L.orc_precoder.argtypes = [F32P, U32, U32, U32, F32P]
        L.orc_equalize.argtypes = [F32P, F32P, U32, U32, U32, U32, ctypes.c_int, U64, U64, U64, U32,
                                   U16P, F32P, U8P, U64, U64, U8P]
        L.orc_precode.argtypes = [F32P, F32P, U32, U32, U32, U32, U32, U32, F32P]
        L.orc_ldpc_sizes.argtypes = [U64, ctypes.c_int, ctypes.c_double, ctypes.c_int, U64, ctypes.c_int,
                                     ctypes.POINTER(U64), ctypes.POINTER(U64), ctypes.POINTER(U64)]
        L.orc_slot_uplink_cpu.restype = ctypes.c_int
        L.orc_slot_uplink_cpu.argtypes = [VP, ctypes.c_int, U32, U32, U32, U32, U32, U32, U32, ctypes.c_int,
                                          U64, U64, U64, F32P, U8P, U64, F32P, F32P, U16P, U8P, ctypes.c_int]
    return _LIB


def _p(a, t):
    return a.ctypes.data_as(t)


def _c64(a):
    a = np.ascontiguousarray(a, dtype=np.complex64)
    return a


DTYPE_CODE = {np.dtype(np.complex64): 0, np.dtype(np.int16): 1, np.dtype(np.int8): 2, np.dtype(np.float16): 3}


def f2h(x):
    return lib().orc_f2h(float(x))


def zadoff_chu(n):
    out = np.zeros(n, np.complex64)
    lib().orc_zadoff_chu(n, _p(out, F32P))
    return out


def cyclic_shift(seq, alpha):
    seq = _c64(seq)
    out = np.zeros_like(seq)
    lib().orc_cyclic_shift(_p(seq, F32P), _p(out, F32P), seq.size, alpha)
    return out


def pilot_sign(S):
    out = np.zeros(S, np.complex64)
    lib().orc_pilot_sign(S, _p(out, F32P))
    return out


def dmrs_table(S, K):
    out = np.zeros((K, S), np.complex64)
    lib().orc_dmrs_table(S, K, _p(out, F32P))
    return out


def scrambler_seq127():
    out = np.zeros(127, np.uint8)
    lib().orc_scrambler_seq127(_p(out, U8P))
    return out


def scramble_bytes(data):
    data = np.ascontiguousarray(data, dtype=np.uint8)
    batch = data.shape[0] if data.ndim == 2 else 1
    nb = data.shape[-1]
    out = np.zeros_like(data)
    lib().orc_scramble_bytes(_p(out, U8P), _p(data, U8P), nb, batch)
    return out


def gold_seq(c_init, n):
    out = np.zeros(n, np.uint8)
    lib().orc_gold_seq(c_init, n, _p(out, U8P))
    return out


def mod_table(Qm):
    out = np.zeros(1 << Qm, np.complex64)
    lib().orc_mod_table(Qm, _p(out, F32P))
    return out


def modulate(bits_bytes, S, Qm, pilot_spacing=0, pilot_table=None):
    bits_bytes = np.ascontiguousarray(bits_bytes, dtype=np.uint8)
    K, in_bytes = bits_bytes.shape
    out = np.zeros((K, S), np.complex64)
    pt = _c64(pilot_table) if pilot_table is not None else np.zeros((K, S), np.complex64)
    lib().orc_modulate(_p(bits_bytes, U8P), _p(out, F32P), in_bytes, S, K, Qm, pilot_spacing, _p(pt, F32P))
    return out


def demod(Qm, x):
    x = np.asarray(x, np.complex64).ravel()
    out = np.zeros((x.size, Qm), np.uint16)
    L = lib()
    for i, v in enumerate(x):
        L.orc_demod(Qm, float(v.real), float(v.imag), _p(out[i], U16P))
    return out.view(np.float16)


def uplink_fft(iq, N, S, start):
    """iq: [M][N] complex64, or [M][N][2] int16/int8/float16."""
    iq = np.ascontiguousarray(iq)
    M = iq.shape[0]
    out = np.zeros((M, S), np.complex64)
    lib().orc_uplink_fft(iq.ctypes.data, DTYPE_CODE[iq.dtype], M, N, S, start, _p(out, F32P))
    return out


def pilot_fft(iq, N, S, start, K, sg, ue_start, psign, csi=None):
    iq = np.ascontiguousarray(iq)
    M = iq.shape[0]
    G = (S + sg - 1) // sg
    if csi is None:
        csi = np.zeros((G, M, K), np.complex64)
    psign = _c64(psign)
    lib().orc_pilot_fft(iq.ctypes.data, DTYPE_CODE[iq.dtype], M, N, S, start, K, sg, ue_start,
                        _p(psign, F32P), _p(csi, F32P))
    return csi


def ifft_downlink(x, out_dtype):
    """x: [M][N] complex64 -> [M][N][2] of out_dtype (int16, int8, float16) or complex64."""
    x = _c64(x)
    M, N = x.shape
    code = DTYPE_CODE[np.dtype(out_dtype)]
    if code == 0:
        out = np.zeros((M, N), np.complex64)
    else:
        out = np.zeros((M, N, 2), out_dtype)
    lib().orc_ifft_downlink(_p(x, F32P), M, N, code, out.ctypes.data)
    return out


def zf(csi, S=None, sg=16, with_cond=False):
    csi = _c64(csi)
    G, M, K = csi.shape
    if S is None:
        S = G * sg
    W = np.zeros_like(csi)
    cond = np.zeros(G, np.float64)
    bad = lib().orc_zf(_p(csi, F32P), G, M, K, S, sg, _p(W, F32P), _p(cond, F64P))
    if with_cond:
        return W, cond, bad
    return W


def precoder(W):
    W = _c64(W)
    G, M, K = W.shape
    P = np.zeros((G, K, M), np.complex64)
    lib().orc_precoder(_p(W, F32P), G, M, K, _p(P, F32P))
    return P


def equalize(W, y, sg, Qm, cb_size, cb_stride, zeros, cb_blocks=1, seq=None, seq_user_stride=0, llr=None):
    W = _c64(W)
    y = _c64(y)
    G, M, K = W.shape
    S = y.shape[1]
    row = cb_stride * cb_blocks
    if llr is None:
        llr = np.zeros((K, row), np.uint16)
    x = np.zeros((K, S), np.complex64)
    if seq is None:
        seq = np.zeros(1, np.uint8)
    seq = np.ascontiguousarray(seq, dtype=np.uint8)
    seq_len = seq.size if seq_user_stride == 0 else seq_user_stride
    n_valid = min(S * Qm, cb_size * cb_blocks)
    hard = np.zeros((K, (n_valid + 7) // 8), np.uint8)
    lib().orc_equalize(_p(W, F32P), _p(y, F32P), K, M, S, sg, Qm, cb_size, cb_stride, zeros, cb_blocks,
                       _p(llr, U16P), _p(x, F32P), _p(seq, U8P), seq_len, seq_user_stride, _p(hard, U8P))
    return llr.view(np.float16), x, hard


def precode(P, s, sg, N, start):
    P = _c64(P)
    s = _c64(s)
    G, K, M = P.shape
    S = s.shape[1]
    out = np.zeros((M, N), np.complex64)
    lib().orc_precode(_p(P, F32P), _p(s, F32P), M, K, S, sg, N, start, _p(out, F32P))
    return out


def ldpc_sizes(S, Qm, rate=1.0 / 3.0, base_graph=1, pilot_spacing=0, downlink=False):
    e, p, d = U64(), U64(), U64()
    lib().orc_ldpc_sizes(S, Qm, rate, base_graph, pilot_spacing, int(downlink),
                         ctypes.byref(e), ctypes.byref(p), ctypes.byref(d))
    return e.value, p.value, d.value


def slot_uplink_cpu(iq, P, U, K, N, S, sg, Qm, cb_size, cb_stride, zeros, psign, seq, threads=0):
    """FP32 OpenMP host baseline for one uplink slot.  iq: [P+U][M][N](...)"""
    iq = np.ascontiguousarray(iq)
    M = iq.shape[1]
    G = (S + sg - 1) // sg
    csi = np.zeros((G, M, K), np.complex64)
    y = np.zeros((U, M, S), np.complex64)
    llr = np.zeros((U, K, cb_stride), np.uint16)
    n_valid = min(S * Qm, cb_size)
    hard = np.zeros((U, K, (n_valid + 7) // 8), np.uint8)
    psign = _c64(psign)
    seq = np.ascontiguousarray(seq, dtype=np.uint8)
    bad = lib().orc_slot_uplink_cpu(iq.ctypes.data, DTYPE_CODE[iq.dtype], P, U, M, K, N, S, sg, Qm,
                                    cb_size, cb_stride, zeros, _p(psign, F32P), _p(seq, U8P), seq.size,
                                    _p(csi, F32P), _p(y, F32P), _p(llr, U16P), _p(hard, U8P), threads)
    return llr.view(np.float16), hard, csi, bad
