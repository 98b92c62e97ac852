"""Per-slot stage runner over the C ABI (mb_slot_*): the single-GPU
replacement of BandProcess::process (baseband/process.cc:134-225)."""
import ctypes

import torch

from . import _lib
from ._lib import LIB, check
from .ops import _dev, _stream

_PREC = {"fp32": _lib.MB_ZF_FP32, "mixed": _lib.MB_ZF_MIXED, "fp64": _lib.MB_ZF_FP64}
_IQ = {"c64": _lib.MB_IQ_C32, "int16": _lib.MB_IQ_I16, "int8": _lib.MB_IQ_I8, "f16": _lib.MB_IQ_F16}
_SCR = {"lfsr127": _lib.MB_SCR_LFSR127, "gold": _lib.MB_SCR_GOLD}


class UplinkSlot:
    """Runs one uplink slot of a cell: pilot FFT -> ZF -> (FFT -> equalize)
    per batch of uplink symbols.  cfg is a datagen.CellConfig (or anything
    with the same fields)."""

    def __init__(self, cfg, precision="fp32", sym_batch=4, use_graph=False, D=0, out_dtype="f16",
                 ns_iters=2, cond_threshold=1e4):
        cb, zeros, stride = cfg.ldpc()
        self.cfg = cfg
        self.cb_size, self.zeros, self.cb_stride = cb, zeros, stride
        self.n_valid = min(cfg.S * cfg.Qm, cb)
        self.hrow = (self.n_valid + 7) // 8
        d = _lib.MbCellDesc(cfg.M, cfg.K, cfg.N, cfg.S, cfg.sg, cfg.Qm, cfg.P, cfg.U, D,
                            _IQ[cfg.iq_dtype], cb, stride, zeros, _PREC[precision], ns_iters,
                            cond_threshold, _SCR[cfg.scrambler], cfg.c_init, _IQ[out_dtype],
                            sym_batch, int(use_graph))
        h = ctypes.c_void_p()
        check(LIB.mb_slot_create(ctypes.byref(d), ctypes.byref(h)), "mb_slot_create")
        self._h = h
        self.D = D
        self.llr = torch.zeros(cfg.U, cfg.K, stride, dtype=torch.float16, device="cuda")
        self.hard = torch.zeros(cfg.U, cfg.K, self.hrow, dtype=torch.uint8, device="cuda")
        self.status = torch.zeros(cfg.G, dtype=torch.int32, device="cuda")

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and LIB is not None:  # LIB is None once the interpreter is shutting down
            LIB.mb_slot_destroy(h)
            self._h = None

    def __call__(self, iq, llr=None, hard=None, stream=None):
        llr = self.llr if llr is None else llr
        hard = self.hard if hard is None else hard
        check(LIB.mb_slot_uplink(self._h, _dev(iq, "iq"), _dev(llr, "llr"), _dev(hard, "hard"),
                                 _dev(self.status, "status"), _stream(stream)), "mb_slot_uplink")
        return llr, hard

    def downlink(self, symbols, out, stream=None):
        check(LIB.mb_slot_downlink(self._h, _dev(symbols, "symbols"), _dev(out, "out"), _stream(stream)),
              "mb_slot_downlink")
        return out

    def downlink_bits(self, bits, out, stream=None):
        """The downlink from encoded bits [D][K][in_bytes] (uint8): modulate,
        precode, inverse FFT (mb_slot_downlink_bits)."""
        check(LIB.mb_slot_downlink_bits(self._h, _dev(bits, "bits"), bits.shape[-1], _dev(out, "out"),
                                        _stream(stream)), "mb_slot_downlink_bits")
        return out

    def set_ldpc(self, code, max_iter=8):
        """Attach an ops.Ldpc whose code block is the cell's (None detaches)."""
        check(LIB.mb_slot_set_ldpc(self._h, code._h if code is not None else None, max_iter), "mb_slot_set_ldpc")
        self._ldpc = code  # not owned by the library: keep it alive

    def decode(self, llr=None, out=None, stream=None):
        """LDPC decode + descramble of the last uplink's LLR rows:
        [U][K][kb Z / 8] uint8 (mb_slot_decode)."""
        llr = self.llr if llr is None else llr
        code = self._ldpc
        if out is None:
            out = torch.zeros(self.cfg.U, self.cfg.K, code.info_bytes, dtype=torch.uint8, device="cuda")
        check(LIB.mb_slot_decode(self._h, _dev(llr, "llr"), _dev(out, "decoded"), _stream(stream)),
              "mb_slot_decode")
        return out

    def downlink_info(self, info, out, stream=None):
        """The downlink from information bits [D][K][kb Z / 8] (uint8):
        scramble, LDPC-encode, modulate, precode, inverse FFT
        (mb_slot_downlink_info; needs set_ldpc)."""
        check(LIB.mb_slot_downlink_info(self._h, _dev(info, "info"), _dev(out, "out"), _stream(stream)),
              "mb_slot_downlink_info")
        return out

    def set_zf_init(self, net):
        """Mixed ZF from the learned polynomial initial iterate of `net` (a
        learned.MLP with 6 inputs and 4 outputs); None: the exact inverse.
        Status 3 then marks groups solved from the learned iterate."""
        check(LIB.mb_slot_set_zf_init(self._h, net._h if net is not None else None), "mb_slot_set_zf_init")
        self._zf_net = net  # not owned by the library: keep it alive

    def timing(self, max_calls):
        """Record per-stage CUDA events for the next max_calls slots."""
        check(LIB.mb_slot_timing(self._h, max_calls), "mb_slot_timing")

    def stage_ms(self):
        """Summed stage times of the recorded calls: dict of ms and counts."""
        out = (ctypes.c_double * 8)()
        check(LIB.mb_slot_stage_ms(self._h, out), "mb_slot_stage_ms")
        keys = ["pilot_fft", "zf", "uplink_fft", "equalize", "slot", "n_fft", "n_eq", "calls"]
        return dict(zip(keys, list(out)))

    def buffers(self):
        """(W [G, M, K], precoder [G, K, M]) as torch views of the slot's buffers."""
        c, p = ctypes.c_void_p(), ctypes.c_void_p()
        check(LIB.mb_slot_buffers(self._h, ctypes.byref(c), ctypes.byref(p)), "mb_slot_buffers")
        cfg = self.cfg
        n = cfg.G * cfg.M * cfg.K
        W = _wrap(c.value, n).view(cfg.G, cfg.M, cfg.K)
        P = _wrap(p.value, n).view(cfg.G, cfg.K, cfg.M)
        return W, P


def _wrap(ptr, n):
    """A complex64 torch view of n elements of library-owned device memory."""
    class _Holder:
        pass
    h = _Holder()
    h.__cuda_array_interface__ = {"shape": (n,), "typestr": "<c8", "data": (ptr, False), "version": 3}
    return torch.as_tensor(h, device="cuda")


class SlotPipeline:
    """Slots from host buffers through the single-GPU pipeline (mb_pipe_*):
    submit() queues one slot (samples in, LLRs and hard bits out, all host
    tensors, pinned for overlap) and returns a ticket; wait(ticket) returns
    once that slot's results are in host memory.  depth slots are in flight:
    the copies of neighbouring slots overlap each slot's kernels."""

    def __init__(self, cfg, precision="mixed", sym_batch=12, depth=2, ns_iters=2, cond_threshold=1e4,
                 use_graph=True):
        cb, zeros, stride = cfg.ldpc()
        self.cfg = cfg
        self.cb_size, self.zeros, self.cb_stride = cb, zeros, stride
        self.hrow = (min(cfg.S * cfg.Qm, cb) + 7) // 8
        d = _lib.MbCellDesc(cfg.M, cfg.K, cfg.N, cfg.S, cfg.sg, cfg.Qm, cfg.P, cfg.U, 0,
                            _IQ[cfg.iq_dtype], cb, stride, zeros, _PREC[precision], ns_iters,
                            cond_threshold, _SCR[cfg.scrambler], cfg.c_init, _IQ["f16"],
                            sym_batch, int(use_graph))
        h = ctypes.c_void_p()
        check(LIB.mb_pipe_create(ctypes.byref(d), depth, ctypes.byref(h)), "mb_pipe_create")
        self._h = h
        a, b, c = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        check(LIB.mb_pipe_io_bytes(h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)), "mb_pipe_io_bytes")
        self.iq_bytes, self.llr_bytes, self.hard_bytes = a.value, b.value, c.value

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and LIB is not None:  # LIB is None once the interpreter is shutting down
            LIB.mb_pipe_destroy(h)
            self._h = None

    def host_outputs(self):
        """Pinned host tensors for one slot's LLRs and hard bits."""
        cfg = self.cfg
        llr = torch.empty(cfg.U, cfg.K, self.cb_stride, dtype=torch.float16).pin_memory()
        hard = torch.empty(cfg.U, cfg.K, self.hrow, dtype=torch.uint8).pin_memory()
        return llr, hard

    def submit(self, iq, llr, hard=None):
        for t, name, n in ((iq, "iq", self.iq_bytes), (llr, "llr", self.llr_bytes),
                           (hard, "hard", self.hard_bytes)):
            if t is None and name == "hard":
                continue
            if t.is_cuda or not t.is_contiguous() or t.numel() * t.element_size() != n:
                raise ValueError(f"{name} must be a contiguous host tensor of {n} bytes")
        ticket = ctypes.c_uint64()
        check(LIB.mb_pipe_submit(self._h, ctypes.c_void_p(iq.data_ptr()), ctypes.c_void_p(llr.data_ptr()),
                                 ctypes.c_void_p(hard.data_ptr()) if hard is not None else None,
                                 ctypes.byref(ticket)), "mb_pipe_submit")
        return ticket.value

    def wait(self, ticket, timeout_ms=None):
        """True once slot `ticket` is done; False if timeout_ms ran out first."""
        r = LIB.mb_pipe_wait(self._h, ticket, 0xFFFFFFFF if timeout_ms is None else int(timeout_ms))
        if r == _lib.MB_TIMEOUT:
            return False
        check(r, "mb_pipe_wait")
        return True

    def set_zf_init(self, net):
        """The pipeline's slots take the learned initial iterate of `net`
        (UplinkSlot.set_zf_init); None: the exact inverse."""
        check(LIB.mb_pipe_set_zf_init(self._h, net._h if net is not None else None), "mb_pipe_set_zf_init")
        self._zf_net = net

    def timer_start(self):
        """Device timer from the next submitted slot's sample copy on."""
        check(LIB.mb_pipe_timer_start(self._h), "mb_pipe_timer_start")

    def timer_ms(self):
        """Device ms from the timer's start to the last submitted slot's results."""
        ms = ctypes.c_double()
        check(LIB.mb_pipe_timer_ms(self._h, ctypes.byref(ms)), "mb_pipe_timer_ms")
        return ms.value
