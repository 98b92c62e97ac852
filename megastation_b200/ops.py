"""Operator objects mirroring the reference's src/operators API over the C ABI.

Same class names, constructor arguments, call signatures and error
behaviour as MegaStation's operators (shape mismatches raise), with torch
CUDA tensors in place of the reference's `Matrix` views.  Tensor shapes are
written slowest-first; the reference's Matrix dims are fastest-first
(matrix.h:95-117), so `Matrix(sizeof(Complex), ofdm, bs)` is a [bs, ofdm]
tensor here.  All compute runs in libmegastation_b200.so; nothing here
computes on the host.
"""
import ctypes

import torch

from . import _lib
from ._lib import LIB, check

_IQ_CODE = {
    torch.complex64: _lib.MB_IQ_C32,
    torch.int16: _lib.MB_IQ_I16,
    torch.int8: _lib.MB_IQ_I8,
    torch.float16: _lib.MB_IQ_F16,
}


def _stream(stream):
    if stream is None:
        return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    if isinstance(stream, torch.cuda.Stream):
        return ctypes.c_void_p(stream.cuda_stream)
    return ctypes.c_void_p(int(stream))


def _dev(t, name, dtype=None):
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")
    if dtype is not None and t.dtype != dtype:
        raise ValueError(f"{name} must be {dtype}, got {t.dtype}")
    return ctypes.c_void_p(t.data_ptr())


def _iq(t, name, M, N):
    """IQ tensor: [..., M, N] complex64 or [..., M, N, 2] int16/int8/float16."""
    if t.dtype not in _IQ_CODE:
        raise ValueError(f"{name}: unsupported dtype {t.dtype}")
    code = _IQ_CODE[t.dtype]
    shape = tuple(t.shape) if code == _lib.MB_IQ_C32 else tuple(t.shape[:-1])
    if code != _lib.MB_IQ_C32 and t.shape[-1] != 2:
        raise ValueError(f"{name}: integer IQ needs a trailing (I, Q) dimension")
    if len(shape) < 2 or shape[-2:] != (M, N):
        raise ValueError(f"{name}: expected [..., {M}, {N}] samples, got {tuple(t.shape)}")
    n_sym = 1
    for d in shape[:-2]:
        n_sym *= d
    return _dev(t, name), code, n_sym


class _FFTBase:
    def __init__(self, ofdm_start, ofdm_ca, ofdm_num, bs_num, ue_num=0, sc_group=0):
        d = _lib.MbFftDesc(ofdm_start, ofdm_ca, ofdm_num, bs_num, ue_num, sc_group)
        h = ctypes.c_void_p()
        check(LIB.mb_fft_create(ctypes.byref(d), ctypes.byref(h)), type(self).__name__)
        self._h = h
        self.ofdm_start, self.ofdm_ca, self.ofdm_num, self.bs_num = ofdm_start, ofdm_ca, ofdm_num, bs_num
        self.ue_num, self.sc_group = ue_num, sc_group

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and LIB is not None:  # LIB is None once the interpreter is shutting down
            LIB.mb_fft_destroy(h)
            self._h = None


class UplinkFFT(_FFTBase):
    """fft/fft_op.h:50-65: forward FFT + shift gather, [..., M, N] -> [..., M, S]."""

    def __init__(self, ofdm_start, ofdm_ca, ofdm_num, bs_num):
        super().__init__(ofdm_start, ofdm_ca, ofdm_num, bs_num)

    def __call__(self, inp, out, stream=None):
        p, code, n_sym = _iq(inp, "in", self.bs_num, self.ofdm_ca)
        if out.dtype != torch.complex64 or out.numel() != n_sym * self.bs_num * self.ofdm_num:
            raise ValueError("out must hold [..., M, S] complex64")
        check(LIB.mb_fft_uplink(self._h, p, code, n_sym, _dev(out, "out"), _stream(stream)),
              "UplinkFFT")

    def uplink_bf16(self, inp, out, row_pitch, stream=None):
        """Planar BF16 rows out[n_sym][re|im][M][row_pitch] (mb_fft_uplink_bf16)."""
        p, code, n_sym = _iq(inp, "in", self.bs_num, self.ofdm_ca)
        if out.dtype != torch.bfloat16 or out.numel() < n_sym * 2 * self.bs_num * row_pitch:
            raise ValueError("out must hold [n_sym, 2, M, row_pitch] bfloat16")
        check(LIB.mb_fft_uplink_bf16(self._h, p, code, n_sym, _dev(out, "out"), row_pitch, _stream(stream)),
              "UplinkFFT.uplink_bf16")


class PilotFFT(_FFTBase):
    """fft/fft_op.h:93-110: forward FFT + LS pilot estimate into CSI [G, M, K]."""

    def __init__(self, ofdm_start, ofdm_ca, ofdm_num, bs_num, ue_num, sc_group):
        super().__init__(ofdm_start, ofdm_ca, ofdm_num, bs_num, ue_num, sc_group)

    def __call__(self, inp, out, ue_start=0, stream=None):
        p, code, n_sym = _iq(inp, "in", self.bs_num, self.ofdm_ca)
        G = (self.ofdm_num + self.sc_group - 1) // self.sc_group
        if out.dtype != torch.complex64 or out.numel() < G * self.bs_num * self.ue_num:
            raise ValueError("out must hold CSI [G, M, K] complex64")
        check(LIB.mb_fft_pilot(self._h, p, code, n_sym, ue_start, _dev(out, "out"), _stream(stream)),
              "PilotFFT")

    def mixed(self, inp, out, ue_start=0, stream=None):
        """The same estimate with the tensor-core FFT (mb_fft_pilot_mixed)."""
        p, code, n_sym = _iq(inp, "in", self.bs_num, self.ofdm_ca)
        G = (self.ofdm_num + self.sc_group - 1) // self.sc_group
        if out.dtype != torch.complex64 or out.numel() < G * self.bs_num * self.ue_num:
            raise ValueError("out must hold CSI [G, M, K] complex64")
        check(LIB.mb_fft_pilot_mixed(self._h, p, code, n_sym, ue_start, _dev(out, "out"), _stream(stream)),
              "PilotFFT.mixed")


class DownlinkIFFT(_FFTBase):
    """fft/fft_op.h:112-120: inverse FFT + quantise, [..., M, N] c64 -> [..., M, N, 2]."""

    def __init__(self, ofdm_start, ofdm_ca, ofdm_num, bs_num):
        super().__init__(ofdm_start, ofdm_ca, ofdm_num, bs_num)

    def __call__(self, inp, out, stream=None):
        if inp.dtype != torch.complex64 or inp.shape[-2:] != (self.bs_num, self.ofdm_ca):
            raise ValueError("in must be [..., M, N] complex64")
        n_sym = inp.numel() // (self.bs_num * self.ofdm_ca)
        if out.dtype not in _IQ_CODE:
            raise ValueError(f"unsupported output dtype {out.dtype}")
        code = _IQ_CODE[out.dtype]
        per = 1 if code == _lib.MB_IQ_C32 else 2
        if out.numel() != inp.numel() * per:
            raise ValueError("out size mismatch")
        check(LIB.mb_ifft_downlink(self._h, _dev(inp, "in"), n_sym, _dev(out, "out"), code,
                                   _stream(stream)), "DownlinkIFFT")

    def mixed(self, inp, out, stream=None):
        """Mixed-precision inverse FFT (mb_ifft_downlink_mixed): inp
        [..., M, N] complex64 or [..., M, N, 2] float16 spectra; at N = 4096
        with int16 / int8 / float16 outputs on the tensor cores."""
        ptr, in_code, n_sym = _iq(inp, "in", self.bs_num, self.ofdm_ca)
        if in_code not in (_lib.MB_IQ_C32, _lib.MB_IQ_F16):
            raise ValueError("in must be complex64 or float16 pairs")
        if out.dtype not in _IQ_CODE:
            raise ValueError(f"unsupported output dtype {out.dtype}")
        code = _IQ_CODE[out.dtype]
        per = 1 if code == _lib.MB_IQ_C32 else 2
        if out.numel() != n_sym * self.bs_num * self.ofdm_ca * per:
            raise ValueError("out size mismatch")
        check(LIB.mb_ifft_downlink_mixed(self._h, ptr, in_code, n_sym, _dev(out, "out"), code, _stream(stream)),
              "DownlinkIFFT.mixed")


class Beamform:
    """beamform/beamform.h:27-84: zero-forcing detector and precoder."""

    def __init__(self, num_bs, num_ue, batch_count, precision=_lib.MB_ZF_FP32, ns_iters=2,
                 cond_threshold=1e4, init_net=None):
        h = ctypes.c_void_p()
        check(LIB.mb_zf_create(num_bs, num_ue, batch_count, ctypes.byref(h)), "Beamform")
        self._h = h
        self.num_bs, self.num_ue, self.batch_count = num_bs, num_ue, batch_count
        self.opts = _lib.MbZfOpts(precision, ns_iters, cond_threshold, 0)
        self._net = None
        if init_net is not None:
            self.set_init_net(init_net)

    def set_init_net(self, net):
        """The mixed ZF starts Newton-Schulz from the learned polynomial
        iterate of `net` (a learned.MLP with 6 inputs and 4 outputs); None
        returns to the exact inverse."""
        check(LIB.mb_zf_set_init_net(self._h, net._h if net is not None else None), "Beamform.set_init_net")
        self._net = net  # the library does not own it: keep it alive
        self.opts.init = 1 if net is not None else 0

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and LIB is not None:  # LIB is None once the interpreter is shutting down
            LIB.mb_zf_destroy(h)
            self._h = None

    def _check_csi(self, csi):
        if csi.dtype != torch.complex64 or csi.shape[-2:] != (self.num_bs, self.num_ue):
            raise ValueError(f"csi must be [G, {self.num_bs}, {self.num_ue}] complex64")
        batch = csi.shape[0] if csi.dim() == 3 else 1
        if batch > self.batch_count:
            # beamform.cu:144-152
            raise ValueError(f"Batch size {batch} exceeds the maximum batch size {self.batch_count}")
        return batch

    def beamform_uplink(self, csi, S=None, sc_group=16, status=None, cond=None, stream=None):
        batch = self._check_csi(csi)
        if S is None:
            S = batch * sc_group
        st = _dev(status, "status", torch.int32) if status is not None else None
        cd = _dev(cond, "cond", torch.float32) if cond is not None else None
        check(LIB.mb_zf_uplink(self._h, _dev(csi, "csi"), batch, S, sc_group, ctypes.byref(self.opts),
                               st, cd, _stream(stream)), "Beamform.beamform_uplink")

    def beamformer(self, csi, precode, S=None, sc_group=16, stream=None):
        batch = self._check_csi(csi)
        if precode.shape[0 if precode.dim() == 3 else -3:] != (batch, self.num_ue, self.num_bs) and \
                precode.numel() != csi.numel():
            raise ValueError("Csi & Precode mismatch")
        self.beamform_uplink(csi, S, sc_group, stream=stream)
        Beamform.beamform_downlink(csi, precode, stream)

    @staticmethod
    def beamform_downlink(csi, precode, stream=None):
        batch = csi.shape[0] if csi.dim() == 3 else 1
        M, K = csi.shape[-2], csi.shape[-1]
        if precode.numel() != csi.numel():
            raise ValueError("Csi & Precode mismatch")
        if precode.shape[-2:] != (K, M):
            raise ValueError("Precode dimension mismatch")
        check(LIB.mb_zf_precoder(_dev(csi, "csi"), _dev(precode, "precode"), M, K, batch,
                                 _stream(stream)), "Beamform.beamform_downlink")


class Scrambler:
    """scrambler/scrambler.h:32-75 plus the descrambling sequence object."""

    def __init__(self, mode=_lib.MB_SCR_LFSR127, c_init=0, num_ue=1, num_bits=0):
        h = ctypes.c_void_p()
        check(LIB.mb_scrambler_create(mode, c_init, num_ue, num_bits, ctypes.byref(h)), "Scrambler")
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and LIB is not None:  # LIB is None once the interpreter is shutting down
            LIB.mb_scrambler_destroy(h)
            self._h = None

    @staticmethod
    def scrambler(out, inp, stream=None):
        if out.dtype != torch.uint8 or inp.dtype != torch.uint8 or out.shape != inp.shape:
            raise ValueError("Input and output mismatch")
        nb = out.shape[-1]
        batch = out.numel() // nb if nb else 0
        check(LIB.mb_scramble(_dev(out, "out"), _dev(inp, "in"), nb, batch, _stream(stream)),
              "Scrambler.scrambler")


class Ldpc:
    """ldpc/encoder.h:48-75 and decoder.h:28-87 (the reference's cuPHY
    LDPCEncoder / LDPCDecoder) over a caller-supplied base graph: entries
    [n][3] of (row, col, shift) with the NR block structure, kb information
    columns, lifting size Z, parity_nodes block rows used.  Bits are packed
    MSB first; LLRs are FP16 rows that start with the 2Z punctured ones."""

    def __init__(self, entries, kb, Z, parity_nodes, max_batch=64):
        import numpy as np
        e = np.asarray(entries).reshape(-1, 3)
        cols = [np.ascontiguousarray(e[:, i], dtype=np.uint16) for i in range(3)]
        g = _lib.MbLdpcGraph(kb, int(e[:, 0].max()) + 1, len(e), *[c.ctypes.data for c in cols])
        h = ctypes.c_void_p()
        check(LIB.mb_ldpc_create(ctypes.byref(g), Z, parity_nodes, max_batch, ctypes.byref(h)), "Ldpc")
        self._h = h
        self.kb, self.Z, self.mb = kb, Z, parity_nodes
        self.info_bytes = (kb * Z + 7) // 8
        self.cw_bits = (kb - 2 + parity_nodes) * Z
        self.n_llr = (kb + parity_nodes) * Z

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and LIB is not None:  # LIB is None once the interpreter is shutting down
            LIB.mb_ldpc_destroy(h)
            self._h = None

    def encode(self, info, out=None, stream=None):
        """info [B][>= kb Z / 8] uint8 -> codewords [B][>= cw_bits / 8] uint8."""
        if out is None:
            out = torch.zeros(info.shape[0], (self.cw_bits + 7) // 8, dtype=torch.uint8, device=info.device)
        check(LIB.mb_ldpc_encode(self._h, _dev(info, "info", torch.uint8), info.stride(0),
                                 _dev(out, "codewords", torch.uint8), out.stride(0), info.shape[0],
                                 _stream(stream)), "Ldpc.encode")
        return out

    def decode(self, llr, max_iter=8, out=None, stream=None):
        """llr [B][>= (kb + mb) Z] float16 -> information bits [B][kb Z / 8] uint8."""
        if out is None:
            out = torch.zeros(llr.shape[0], self.info_bytes, dtype=torch.uint8, device=llr.device)
        check(LIB.mb_ldpc_decode(self._h, _dev(llr, "llr", torch.float16), llr.stride(0),
                                 _dev(out, "out", torch.uint8), out.stride(0), llr.shape[0], max_iter,
                                 _stream(stream)), "Ldpc.decode")
        return out


class Equalize:
    """sgemv/equalize.h:25-74: equalize + demodulate (+ descrambled hard bits)."""

    @staticmethod
    def equalize(csi, bsVec, ueVec, csi_skip, mod_order, cb_size, zeros, cb_blocks=1,
                 hard=None, scrambler=None, x=None, stream=None):
        if csi.dtype != torch.complex64 or bsVec.dtype != torch.complex64:
            raise ValueError("csi and bsVec must be complex64")
        M, K = csi.shape[-2], csi.shape[-1]
        S = bsVec.shape[-1]
        if bsVec.shape[-2] != M:
            raise ValueError("bsVec must be [..., M, S]")
        n_sym = bsVec.numel() // (M * S)
        if ueVec.dtype != torch.float16:
            raise ValueError("ueVec must be float16")
        cb_stride = ueVec.shape[-1]  # equalize.cu:57-63 (ueVec.stride(1))
        if ueVec.numel() != n_sym * K * cb_blocks * cb_stride:
            raise ValueError("ueVec must be [n_sym, K*cb_blocks, cb_stride]")
        hp = _dev(hard, "hard", torch.uint8) if hard is not None else None
        sp = scrambler._h if scrambler is not None else None
        xp = _dev(x, "x", torch.complex64) if x is not None else None
        check(LIB.mb_equalize(_dev(csi, "csi"), _dev(bsVec, "bsVec"), K, M, S, csi_skip, n_sym,
                              mod_order, cb_size, cb_stride, zeros, cb_blocks, _dev(ueVec, "ueVec"),
                              hp, sp, xp, _stream(stream)), "Equalize.equalize")


    @staticmethod
    def equalize_tc(csi, bsVec, ueVec, csi_skip, mod_order, cb_size, zeros, cb_blocks=1,
                    hard=None, scrambler=None, x=None, stream=None):
        """Mixed-precision variant on the tensor cores (BF16 W and y, FP32
        accumulation); scratch is allocated here by torch, outside the library."""
        M, K = csi.shape[-2], csi.shape[-1]
        S = bsVec.shape[-1]
        n_sym = bsVec.numel() // (M * S)
        img, ylp = _lib.U64(), _lib.U64()
        check(LIB.mb_equalize_tc_scratch(K, M, S, csi_skip, n_sym, ctypes.byref(img), ctypes.byref(ylp)),
              "mb_equalize_tc_scratch")
        s_img = torch.empty(img.value, dtype=torch.uint8, device=csi.device)
        s_ylp = torch.empty(ylp.value, dtype=torch.uint8, device=csi.device)
        cb_stride = ueVec.shape[-1]
        if ueVec.numel() != n_sym * K * cb_blocks * cb_stride:
            raise ValueError("ueVec must be [n_sym, K*cb_blocks, cb_stride]")
        hp = _dev(hard, "hard", torch.uint8) if hard is not None else None
        sp = scrambler._h if scrambler is not None else None
        xp = _dev(x, "x", torch.complex64) if x is not None else None
        check(LIB.mb_equalize_tc(_dev(csi, "csi"), _dev(bsVec, "bsVec"), K, M, S, csi_skip, n_sym, mod_order,
                                 cb_size, cb_stride, zeros, cb_blocks, _dev(ueVec, "ueVec"), hp, sp, xp,
                                 _dev(s_img, "img"), _dev(s_ylp, "ylp"), _stream(stream)), "Equalize.equalize_tc")


def device_error(clear=True):
    """Error bits of bounded device waits that gave up (0 = none)."""
    v = ctypes.c_int()
    check(LIB.mb_device_error(ctypes.byref(v), int(clear)), "mb_device_error")
    return v.value


class Precode:
    """sgemv/precode.h:24-62: precode + FFT-shift scatter into N-point rows."""

    @staticmethod
    def precode(precoded, ueVec, bsVec, precode_skip, bs_start, stream=None):
        K, M = precoded.shape[-2], precoded.shape[-1]
        S = ueVec.shape[-1]
        if ueVec.shape[-2] != K:
            raise ValueError("ueVec must be [..., K, S]")
        n_sym = ueVec.numel() // (K * S)
        N = bsVec.shape[-1]  # precode.cu:64 (bsVec.stride(1))
        if bsVec.numel() != n_sym * M * N:
            raise ValueError("bsVec must be [n_sym, M, N]")
        check(LIB.mb_precode(_dev(precoded, "precoded"), _dev(ueVec, "ueVec"), M, K, S, precode_skip,
                             N, bs_start, n_sym, _dev(bsVec, "bsVec"), _stream(stream)),
              "Precode.precode")


    @staticmethod
    def precode_tc(precoded, ueVec, z, precode_skip, bs_start, scratch=None, stream=None):
        """Mixed-precision precode on the tensor cores (mb_precode_tc):
        z [n_sym, M, N, 2] float16 gets the data bins; the other bins are
        left as they are.  scratch: a uint8 CUDA tensor of at least
        mb_precode_tc_scratch bytes (allocated here when None)."""
        K, M = precoded.shape[-2], precoded.shape[-1]
        S = ueVec.shape[-1]
        n_sym = ueVec.numel() // (K * S)
        if z.dtype != torch.float16 or z.shape[-1] != 2 or z.shape[-3] != M or z.numel() % (n_sym * M * 2):
            raise ValueError("z must be [n_sym, M, N, 2] float16")
        N = z.shape[-2]
        nb = _lib.U64()
        check(LIB.mb_precode_tc_scratch(M, K, S, precode_skip, ctypes.byref(nb)), "mb_precode_tc_scratch")
        if scratch is None:
            scratch = torch.empty(nb.value, dtype=torch.uint8, device=z.device)
        if scratch.numel() < nb.value:
            raise ValueError(f"scratch needs {nb.value} bytes")
        check(LIB.mb_precode_tc(_dev(precoded, "precoded", torch.complex64), _dev(ueVec, "ueVec", torch.complex64),
                                M, K, S, precode_skip, N, bs_start, n_sym, _dev(z, "z"), _dev(scratch, "scratch"),
                                _stream(stream)), "Precode.precode_tc")


class Modulation:
    """modulation/modulation.h:27-90: bits -> QAM with optional DM-RS pilots."""

    @staticmethod
    def modulate(inp, out, mod_order, pilot_spacing=0, pilot_table=None, stream=None):
        K, S = out.shape[-2], out.shape[-1]
        in_bytes = inp.shape[-1]
        pt = _dev(pilot_table, "pilot_table", torch.complex64) if pilot_table is not None else None
        check(LIB.mb_modulate(_dev(inp, "in", torch.uint8), _dev(out, "out", torch.complex64), in_bytes,
                              S, K, mod_order, pilot_spacing, pt, _stream(stream)), "Modulation.modulate")


def pilot_sign(S):
    """Host pilot table p/|p|^2 (fft_op.cu:176-192) as a complex64 CPU tensor."""
    out = torch.zeros(S, dtype=torch.complex64)
    check(LIB.mb_pilot_sign(S, ctypes.c_void_p(out.data_ptr())), "pilot_sign")
    return out


def dmrs_table(S, K):
    out = torch.zeros(K, S, dtype=torch.complex64)
    check(LIB.mb_dmrs_table(S, K, ctypes.c_void_p(out.data_ptr())), "dmrs_table")
    return out


def ldpc_sizes(S, Qm, code_rate=1.0 / 3.0, base_graph=1, pilot_spacing=0, downlink=False):
    e, p, d = _lib.U64(), _lib.U64(), _lib.U64()
    check(LIB.mb_ldpc_sizes(S, Qm, code_rate, base_graph, pilot_spacing, int(downlink),
                            ctypes.byref(e), ctypes.byref(p), ctypes.byref(d)), "ldpc_sizes")
    return e.value, p.value, d.value
