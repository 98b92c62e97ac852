"""The bench's workload arithmetic on CPU: the compulsory bytes of a slot
follow its sample format, and the rotated input slots always exceed the
126 MB L2 so that every timed step reads its samples from HBM."""
import argparse
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


@pytest.fixture(scope="module")
def bench():
    import bench as b
    return b


def _cfg(bench, iq):
    from megastation_b200 import datagen
    return datagen.CellConfig(**{**bench.WORKLOAD, "iq_dtype": iq})


def test_slot_bytes_follow_the_sample_format(bench):
    c8, c16 = _cfg(bench, "int8"), _cfg(bench, "int16")
    samples = c8.symbols * c8.M * c8.N
    # samples in (2 or 4 bytes each) + FP16 LLRs + packed hard bits out
    assert bench.algorithmic_bytes(c16) - bench.algorithmic_bytes(c8) == samples * 2
    cb, _, _ = c8.ldpc()
    n_valid = min(c8.S * c8.Qm, cb)
    out = c8.U * c8.K * (n_valid * 2 + (n_valid + 7) // 8)
    assert bench.algorithmic_bytes(c8) == samples * 2 + out
    assert bench.algorithmic_bytes(c8, b_in=8) == samples * 8 + out


@pytest.mark.parametrize("iq", ["int8", "int16", "c64", "f16"])
def test_rotated_inputs_exceed_l2(bench, iq):
    cfg = _cfg(bench, iq)
    for rotate in (1, 2, 4):
        args = argparse.Namespace(rotate=rotate)
        R = bench.rotation(cfg, args)
        assert R >= max(2, rotate)
        assert R * cfg.symbols * cfg.M * cfg.N * bench.IQ_BYTES[iq] >= 1.25 * 126e6
