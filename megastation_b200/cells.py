"""Batched uneven cells over the C ABI (mb_cells_*): one CUDA graph launch
runs one uplink slot of every cell.  No counterpart in the reference, which
processes one cell per BandProcess (baseband/process.cc:134-225)."""
import ctypes

import torch

from . import _lib
from ._lib import LIB, check
from .ops import _dev, _stream
from .slot import _IQ, _PREC, _SCR


def _ptrs(tensors):
    arr = (ctypes.c_void_p * len(tensors))()
    for i, t in enumerate(tensors):
        arr[i] = None if t is None else _dev(t, "cell buffer")
    return arr


class Cells:
    """cfgs: datagen.CellConfig per cell (shapes may all differ)."""

    def __init__(self, cfgs, precision="mixed", ns_iters=2, cond_threshold=1e4):
        self.cfgs = list(cfgs)
        descs = (_lib.MbCellDesc * len(self.cfgs))()
        self.llr, self.hard, self.status = [], [], []
        for i, cfg in enumerate(self.cfgs):
            cb, zeros, stride = cfg.ldpc()
            n_valid = min(cfg.S * cfg.Qm, cb)
            descs[i] = _lib.MbCellDesc(cfg.M, cfg.K, cfg.N, cfg.S, cfg.sg, cfg.Qm, cfg.P, cfg.U, 0,
                                       _IQ[cfg.iq_dtype], cb, stride, zeros, _PREC[precision], ns_iters,
                                       cond_threshold, _SCR[cfg.scrambler], cfg.c_init, _IQ["f16"],
                                       max(cfg.U, 1), 0)
            self.llr.append(torch.zeros(cfg.U, cfg.K, stride, dtype=torch.float16, device="cuda"))
            self.hard.append(torch.zeros(cfg.U, cfg.K, (n_valid + 7) // 8, dtype=torch.uint8, device="cuda"))
            self.status.append(torch.zeros(cfg.G, dtype=torch.int32, device="cuda"))
        h = ctypes.c_void_p()
        check(LIB.mb_cells_create(descs, len(self.cfgs), ctypes.byref(h)), "mb_cells_create")
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and LIB is not None:  # LIB is None once the interpreter is shutting down
            LIB.mb_cells_destroy(h)
            self._h = None

    def __call__(self, iqs, llr=None, hard=None, stream=None):
        """One slot of every cell; iqs[c] is cell c's [P+U][M][N] samples on
        the device.  Returns the (llr, hard) lists."""
        llr = self.llr if llr is None else llr
        hard = self.hard if hard is None else hard
        check(LIB.mb_cells_uplink(self._h, _ptrs(iqs), _ptrs(llr), _ptrs(hard), _ptrs(self.status),
                                  _stream(stream)), "mb_cells_uplink")
        return llr, hard

    def autotune(self, iqs, reps=20, stream=None):
        """Picks sym_batch, equalizer columns per CTA, the tensor-core FFT's
        CTAs per launch and the mixed ZF's product path per cell class by
        timing the batched slot; returns (per-cell choices, us per slot)."""
        n = len(self.cfgs)
        sb, cols = (ctypes.c_uint32 * n)(), (ctypes.c_uint32 * n)()
        us = ctypes.c_double()
        check(LIB.mb_cells_autotune(self._h, _ptrs(iqs), _ptrs(self.llr), _ptrs(self.hard), reps,
                                    _stream(stream), sb, cols, ctypes.byref(us)), "mb_cells_autotune")
        return self.tuning(), us.value

    def tuning(self):
        n = len(self.cfgs)
        sb, cols, fc, zp = [(ctypes.c_uint32 * n)() for _ in range(4)]
        check(LIB.mb_cells_get_tuning(self._h, sb, cols), "mb_cells_get_tuning")
        check(LIB.mb_cells_get_fft_ctas(self._h, fc), "mb_cells_get_fft_ctas")
        check(LIB.mb_cells_get_zf_path(self._h, zp), "mb_cells_get_zf_path")
        return [{"sym_batch": sb[i], "eq_cols": cols[i], "fft_ctas": fc[i], "zf_path": zp[i]} for i in range(n)]

    def set_tuning(self, choices):
        n = len(self.cfgs)
        sb = (ctypes.c_uint32 * n)(*[c["sym_batch"] for c in choices])
        cols = (ctypes.c_uint32 * n)(*[c["eq_cols"] for c in choices])
        check(LIB.mb_cells_set_tuning(self._h, sb, cols), "mb_cells_set_tuning")
        if all("fft_ctas" in c for c in choices):
            fc = (ctypes.c_uint32 * n)(*[c["fft_ctas"] for c in choices])
            check(LIB.mb_cells_set_fft_ctas(self._h, fc), "mb_cells_set_fft_ctas")
        if all("zf_path" in c for c in choices):
            zp = (ctypes.c_uint32 * n)(*[c["zf_path"] for c in choices])
            check(LIB.mb_cells_set_zf_path(self._h, zp), "mb_cells_set_zf_path")
