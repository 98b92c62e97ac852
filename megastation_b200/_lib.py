"""ctypes binding of libmegastation_b200.so (the C ABI in include/megastation_b200.h).

The shared library is the product: there is no Python or CPU fallback.  If it
is missing or fails to load, importing this module raises.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmegastation_b200.so")

# mb_status
MB_OK = 0
MB_BAD_SHAPE = 1
MB_BAD_ARG = 2
MB_NOT_PD = 3
MB_CUDA_ERROR = 4
MB_TIMEOUT = 5
MB_NO_MEMORY = 6
MB_UNSUPPORTED = 7
MB_TOO_LARGE = 8

# mb_iq_dtype
MB_IQ_C32 = 0
MB_IQ_I16 = 1
MB_IQ_I8 = 2
MB_IQ_F16 = 3

# mb_zf_precision
MB_ZF_FP32 = 0
MB_ZF_MIXED = 1
MB_ZF_FP64 = 2

# mb_scrambler_mode
MB_SCR_LFSR127 = 0
MB_SCR_GOLD = 1

VP = ctypes.c_void_p
U32 = ctypes.c_uint32
U64 = ctypes.c_uint64
I32 = ctypes.c_int
ST = ctypes.c_int


class MbC32(ctypes.Structure):
    _fields_ = [("re", ctypes.c_float), ("im", ctypes.c_float)]


class MbFftDesc(ctypes.Structure):
    _fields_ = [("ofdm_start", U32), ("ofdm_ca", U32), ("ofdm_num", U32),
                ("bs_num", U32), ("ue_num", U32), ("sc_group", U32)]


class MbZfOpts(ctypes.Structure):
    _fields_ = [("precision", U32), ("ns_iters", U32), ("cond_threshold", ctypes.c_float),
                ("init", U32)]


class MbLdpcGraph(ctypes.Structure):
    _fields_ = [("kb", U32), ("rows", U32), ("nnz", U32), ("row", VP), ("col", VP), ("shift", VP)]


class MbCellDesc(ctypes.Structure):
    _fields_ = [("M", U32), ("K", U32), ("N", U32), ("S", U32), ("sg", U32), ("Qm", U32),
                ("P", U32), ("U", U32), ("D", U32), ("iq_dtype", ctypes.c_int32),
                ("cb_size", U64), ("cb_stride", U64), ("zeros", U64),
                ("zf_precision", U32), ("ns_iters", U32), ("cond_threshold", ctypes.c_float),
                ("scrambler_mode", U32), ("c_init", U32), ("out_dtype", ctypes.c_int32),
                ("sym_batch", U32), ("use_graph", U32)]


class MbError(RuntimeError):
    def __init__(self, status, where):
        self.status = status
        super().__init__(f"{where}: {status_str(status)} (mb_status {status})")


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `make -C megastation_b200` "
            "(or __graft_entry__.build()); there is no fallback path")
    lib = ctypes.CDLL(LIB_PATH)
    sigs = {
        "mb_status_str": (ctypes.c_char_p, [ST]),
        "mb_version": (ctypes.c_char_p, []),
        "mb_tables_init": (ST, [I32]),
        "mb_pilot_sign": (ST, [U64, VP]),
        "mb_dmrs_table": (ST, [U64, U64, VP]),
        "mb_ldpc_sizes": (ST, [U64, U32, ctypes.c_double, U32, U64, I32,
                               ctypes.POINTER(U64), ctypes.POINTER(U64), ctypes.POINTER(U64)]),
        "mb_pipe_create": (ST, [ctypes.POINTER(MbCellDesc), U32, ctypes.POINTER(VP)]),
        "mb_pipe_destroy": (ST, [VP]),
        "mb_pipe_io_bytes": (ST, [VP, ctypes.POINTER(U64), ctypes.POINTER(U64), ctypes.POINTER(U64)]),
        "mb_pipe_submit": (ST, [VP, VP, VP, VP, ctypes.POINTER(U64)]),
        "mb_pipe_wait": (ST, [VP, U64, U32]),
        "mb_pipe_set_zf_init": (ST, [VP, VP]),
        "mb_pipe_timer_start": (ST, [VP]),
        "mb_pipe_timer_ms": (ST, [VP, ctypes.POINTER(ctypes.c_double)]),
        "mb_fft_create": (ST, [ctypes.POINTER(MbFftDesc), ctypes.POINTER(VP)]),
        "mb_fft_destroy": (ST, [VP]),
        "mb_fft_uplink": (ST, [VP, VP, I32, U32, VP, VP]),
        "mb_fft_uplink_bf16": (ST, [VP, VP, I32, U32, VP, U32, VP]),
        "mb_fft_pilot": (ST, [VP, VP, I32, U32, U32, VP, VP]),
        "mb_fft_pilot_mixed": (ST, [VP, VP, I32, U32, U32, VP, VP]),
        "mb_ifft_downlink": (ST, [VP, VP, U32, VP, I32, VP]),
        "mb_zf_create": (ST, [U32, U32, U32, ctypes.POINTER(VP)]),
        "mb_zf_destroy": (ST, [VP]),
        "mb_zf_uplink": (ST, [VP, VP, U32, U32, U32, ctypes.POINTER(MbZfOpts), VP, VP, VP]),
        "mb_zf_precoder": (ST, [VP, VP, U32, U32, U32, VP]),
        "mb_zf_set_init_net": (ST, [VP, VP]),
        "mb_zf_init_targets": (ST, [VP, U32, U32, U32, VP, VP, VP, VP]),
        "mb_slot_set_zf_init": (ST, [VP, VP]),
        "mb_scrambler_create": (ST, [I32, U32, U32, U64, ctypes.POINTER(VP)]),
        "mb_scrambler_destroy": (ST, [VP]),
        "mb_equalize": (ST, [VP, VP, U32, U32, U32, U32, U32, U32, U64, U64, U64, U32,
                             VP, VP, VP, VP, VP]),
        "mb_equalize_tc_scratch": (ST, [U32, U32, U32, U32, U32, ctypes.POINTER(U64), ctypes.POINTER(U64)]),
        "mb_equalize_tc": (ST, [VP, VP, U32, U32, U32, U32, U32, U32, U64, U64, U64, U32,
                                VP, VP, VP, VP, VP, VP, VP]),
        "mb_equalize_tc_noalloc": (ST, [VP, VP, U32, U32, U32, U32, U32, U32, U64, U64, U64, U32,
                                        VP, VP, VP, VP, VP]),
        "mb_device_error": (ST, [ctypes.POINTER(ctypes.c_int), I32]),
        "mb_selftest_wait": (ST, [U64, I32, VP]),
        "mb_precode": (ST, [VP, VP, U32, U32, U32, U32, U32, U32, U32, VP, VP]),
        "mb_precode_tc_scratch": (ST, [U32, U32, U32, U32, ctypes.POINTER(U64)]),
        "mb_precode_tc": (ST, [VP, VP, U32, U32, U32, U32, U32, U32, U32, VP, VP, VP]),
        "mb_ifft_downlink_mixed": (ST, [VP, VP, I32, U32, VP, I32, VP]),
        "mb_modulate": (ST, [VP, VP, U64, U64, U64, U32, U32, VP, VP]),
        "mb_scramble": (ST, [VP, VP, U64, U64, VP]),
        "mb_slot_create": (ST, [ctypes.POINTER(MbCellDesc), ctypes.POINTER(VP)]),
        "mb_slot_destroy": (ST, [VP]),
        "mb_slot_uplink": (ST, [VP, VP, VP, VP, VP, VP]),
        "mb_slot_downlink": (ST, [VP, VP, VP, VP]),
        "mb_slot_downlink_bits": (ST, [VP, VP, U64, VP, VP]),
        "mb_slot_set_ldpc": (ST, [VP, VP, U32]),
        "mb_slot_decode": (ST, [VP, VP, VP, VP]),
        "mb_slot_downlink_info": (ST, [VP, VP, VP, VP]),
        "mb_slot_buffers": (ST, [VP, ctypes.POINTER(VP), ctypes.POINTER(VP)]),
        "mb_slot_timing": (ST, [VP, U32]),
        "mb_slot_stage_ms": (ST, [VP, ctypes.POINTER(ctypes.c_double)]),
        "mb_cells_create": (ST, [ctypes.POINTER(MbCellDesc), U32, ctypes.POINTER(VP)]),
        "mb_cells_destroy": (ST, [VP]),
        "mb_cells_uplink": (ST, [VP, VP, VP, VP, VP, VP]),
        "mb_cells_autotune": (ST, [VP, VP, VP, VP, U32, VP, ctypes.POINTER(U32), ctypes.POINTER(U32),
                                   ctypes.POINTER(ctypes.c_double)]),
        "mb_cells_get_tuning": (ST, [VP, ctypes.POINTER(U32), ctypes.POINTER(U32)]),
        "mb_cells_get_fft_ctas": (ST, [VP, ctypes.POINTER(U32)]),
        "mb_cells_set_fft_ctas": (ST, [VP, ctypes.POINTER(U32)]),
        "mb_cells_get_zf_path": (ST, [VP, VP]),
        "mb_ldpc_create": (ST, [VP, U32, U32, U32, VP]),
        "mb_ldpc_destroy": (ST, [VP]),
        "mb_ldpc_encode": (ST, [VP, VP, U64, VP, U64, U32, VP]),
        "mb_ldpc_decode": (ST, [VP, VP, U64, VP, U64, U32, U32, VP]),
        "mb_cells_set_zf_path": (ST, [VP, VP]),
        "mb_cells_set_tuning": (ST, [VP, ctypes.POINTER(U32), ctypes.POINTER(U32)]),
    }
    for name, (res, args) in sigs.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


LIB = _load()


def status_str(status):
    return LIB.mb_status_str(status).decode()


def check(status, where):
    if status != MB_OK:
        raise MbError(status, where)
