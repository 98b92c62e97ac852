"""Pins the CPU oracle to the golden vectors of the reference's own unit tests.

Each case restates one reference test (file:line in the MegaStation tree) with
its shapes, arguments and tolerance; the fixtures under tests/golden/ are the
reference's .data files (see tests/golden/make_golden.py).
"""
import os

import numpy as np
import pytest

from oracle import oracle as orc

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def gold(sub, name, dtype):
    return np.fromfile(os.path.join(GOLD, sub, name + ".data"), dtype=dtype)


def test_zadoff_chu_golden():
    # test/fft/test_fft.cc:10-30
    ref = gold("fft", "zachu", np.complex64)
    out = orc.zadoff_chu(32)[:31]
    np.testing.assert_allclose(out, ref, atol=1e-5)


def test_zadoff_chu_shift_golden():
    # test/fft/test_fft.cc:32-53
    ref = gold("fft", "zachu_shift", np.complex64)
    out = orc.cyclic_shift(orc.zadoff_chu(16), np.float32(np.pi / 4))
    np.testing.assert_allclose(out, ref, atol=1e-5)


def test_pilot_fft_golden():
    # test/fft/test_fft.cc:55-104: ue=4, bs=8, N=32, S=16, sc_group=4, start=8
    iq = gold("fft", "short_in", np.int16).reshape(8, 32, 2)
    ref = gold("fft", "complex_out", np.complex64).reshape(4, 8, 4)
    csi = orc.pilot_fft(iq, N=32, S=16, start=8, K=4, sg=4, ue_start=0, psign=orc.pilot_sign(16))
    np.testing.assert_allclose(csi, ref, atol=1e-4)


def test_uplink_fft_golden():
    # test/fft/test_fft.cc:106-173: bs=8, N=32, S=16, start=8; reference
    # output stored [S][M] by the test
    iq = gold("fft", "fft_in", np.int16).reshape(8, 32, 2)
    ref = gold("fft", "fft_out", np.complex64).reshape(16, 8)
    out = orc.uplink_fft(iq, N=32, S=16, start=8)
    np.testing.assert_allclose(out.T, ref, atol=1e-5)


def test_downlink_ifft_golden_bit_exact():
    # test/fft/test_fft.cc:175-215: int16 output compared with EXPECT_EQ
    x = gold("fft", "ifft_in", np.complex64).reshape(8, 32)
    ref = gold("fft", "ifft_out", np.int16).reshape(8, 32, 2)
    out = orc.ifft_downlink(x, np.int16)
    np.testing.assert_array_equal(out, ref)


def test_beamform_golden():
    # test/beamform/test_beamform.cc:67-95: K=4, M=8, two identical batches
    csi = gold("beamform", "csi_in", np.complex64).reshape(1, 8, 4)
    csi = np.concatenate([csi, csi])
    W = orc.zf(csi, S=32, sg=16)
    P = orc.precoder(W)
    ref_w = gold("beamform", "csi_out", np.complex64).reshape(8, 4)
    ref_p = gold("beamform", "precoder", np.complex64).reshape(4, 8)
    for g in range(2):
        np.testing.assert_allclose(W[g], ref_w, atol=1e-5)
        np.testing.assert_allclose(P[g], ref_p, atol=1e-5)


def test_equalize_golden_bit_exact():
    # test/sgemv/test_sgemv.cc:126-159: K=4, M=8, 16 subcarriers (one group),
    # QPSK, cb_size=32, zeros=0, one code block; FP16 compared with EXPECT_EQ
    W = gold("sgemv", "csi", np.complex64).reshape(1, 8, 4)
    y = gold("sgemv", "bsVec", np.complex64).reshape(16, 8).T.copy()
    ref = gold("sgemv", "equalize", np.uint16).reshape(4, 32)
    llr, _, _ = orc.equalize(W, y, sg=16, Qm=2, cb_size=32, cb_stride=32, zeros=0)
    np.testing.assert_array_equal(llr.view(np.uint16), ref)


def test_precode_golden():
    # test/sgemv/test_sgemv.cc:161-196: M=8, K=4, 16 subcarriers, N=32, start=8
    P = gold("sgemv", "prec", np.complex64).reshape(1, 4, 8)
    s = gold("sgemv", "ueVec", np.complex64).reshape(16, 4).T.copy()
    ref = gold("sgemv", "precoded", np.complex64).reshape(8, 32)
    out = orc.precode(P, s, sg=16, N=32, start=8)
    np.testing.assert_allclose(out, ref, atol=1e-5)


def test_modulate_64qam_round_trip():
    # test/modulation/test_modulation.cc:11-57: bytes 0..63 packed LSB-first,
    # 6 bits per symbol, 4 users; hard decision llr<0 -> 1 recovers them
    vals = np.arange(64, dtype=np.uint8)
    bits = ((vals[:, None] >> np.arange(6)) & 1).astype(np.uint8).ravel()
    packed = np.packbits(bits, bitorder="little")
    inp = np.tile(packed, (4, 1))
    sym = orc.modulate(inp, S=64, Qm=6)
    for u in range(4):
        llr = orc.demod(6, sym[u])
        got = ((llr.astype(np.float32) < 0).astype(np.uint8) << np.arange(6)).sum(1)
        np.testing.assert_array_equal(got, vals)


@pytest.mark.parametrize("Qm", [2, 4, 6, 8])
def test_modulate_demod_round_trip_all_orders(Qm):
    # known answer beyond the reference's 64-QAM test: every table entry
    # demaps to its own bits (demodulation.h:30-67, modulation.cu:22-72)
    n = 1 << Qm
    vals = np.arange(n)
    bits = ((vals[:, None] >> np.arange(Qm)) & 1).astype(np.uint8).ravel()
    packed = np.packbits(bits, bitorder="little")[None, :]
    sym = orc.modulate(packed, S=n, Qm=Qm)[0]
    llr = orc.demod(Qm, sym)
    got = ((llr.astype(np.float32) < 0).astype(np.int64) << np.arange(Qm)).sum(1)
    if Qm == 8:
        # the reference's 256-QAM table (modulation.cu:56-72) and its demapper
        # (demodulation.h:52-65) disagree on every bit: the table maps a first
        # bit of 1 to positive I while the demapper decides 1 for negative I,
        # and likewise for the amplitude bits.  Pinned as found.
        np.testing.assert_array_equal(got, vals ^ 0xFF)
    else:
        np.testing.assert_array_equal(got, vals)
    # unit average power
    assert abs(np.mean(np.abs(orc.mod_table(Qm)) ** 2) - 1.0) < 1e-5


def test_scrambler_involution_and_sequence():
    # test/scrambler/test_scrambler.cc:9-46 (involution) plus a known-answer
    # pin of the LFSR: period 127, 64 ones (maximal-length m-sequence)
    data = np.frombuffer(b"Hello World!\0", np.uint8).copy()
    once = orc.scramble_bytes(data)
    assert not np.array_equal(once, data)
    np.testing.assert_array_equal(orc.scramble_bytes(once), data)
    seq = orc.scrambler_seq127()
    assert seq.sum() == 64
    # x^7 + x^4 + 1 recurrence with state 0x5D (scrambler.cu:24-31)
    s = 0x5D
    for i in range(127):
        fb = (s ^ (s >> 3)) & 1
        assert seq[i] == fb
        s = (s >> 1) | (fb << 6)
    assert s == 0x5D
    rng = np.random.default_rng(0)
    multi = rng.integers(0, 256, (4, 137), dtype=np.uint8)
    np.testing.assert_array_equal(orc.scramble_bytes(orc.scramble_bytes(multi)), multi)


def test_gold_sequence_known_answer():
    # TS 38.211 5.2.1 with c_init = 0: x2 stays zero, so c(n) = x1(n + 1600)
    x1 = np.zeros(1600 + 64 + 31, np.uint8)
    x1[0] = 1
    for n in range(len(x1) - 31):
        x1[n + 31] = x1[n + 3] ^ x1[n]
    np.testing.assert_array_equal(orc.gold_seq(0, 64), x1[1600:1664])
    a, b = orc.gold_seq(0x1234, 256), orc.gold_seq(0x1235, 256)
    assert (a != b).any()


def test_ldpc_sizes_reference_configs():
    # config.cc:84-135 at the reference's own main.cc setting (S=1200, 64-QAM,
    # rate 1/3, BG1): Zc=104 -> E=(22-2+46)*104, punctured 2*Zc
    e, p, d = orc.ldpc_sizes(1200, 6)
    assert (e, p, d) == (66 * 104, 208, 22 * 104)
    e, p, d = orc.ldpc_sizes(3276, 6)
    assert (e, p, d) == (66 * 288, 576, 22 * 288)
