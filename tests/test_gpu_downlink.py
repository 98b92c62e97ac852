"""The downlink of a slot (mb_slot_downlink through the C ABI) against the
CPU oracle end to end: the precoder of the slot's own uplink ZF
(beamform.cu:154-168, beam_utils.cuh:40-80), precoding with the FFT-shift
scatter (precode_kernel.cuh:255-262) and the inverse FFT with its output
quantiser (fft_op.cu:167-174, ifft_callback.cuh:21-59).  The full-slot shape
is 256 antennas x 64 users, N = 4096, S = 3276, 4 pilot + 5 uplink + 5
downlink symbols of 256-QAM at 30 dB over the correlated 8-tap channel, with
complex FP16 and int16 antenna samples out."""
import numpy as np
import pytest
import torch

from oracle import oracle as orc

from slot_oracle import check_uplink, oracle_uplink

pytestmark = pytest.mark.gpu

FULL = dict(M=256, K=64, N=4096, S=3276, sg=16, Qm=8, U=5, snr_db=30.0, channel="tdl", n_taps=8,
            tap_decay=2.0, rho=0.5, seed=5050)
SMALL = dict(M=32, K=8, N=512, S=300, sg=16, Qm=4, U=2, snr_db=25.0, seed=61)


def _downlink_ref(cfg, W, syms, out_dtype):
    P = orc.precoder(W)
    outs = []
    for s in syms:
        z = orc.precode(P, s, cfg.sg, cfg.N, cfg.start)
        outs.append(orc.ifft_downlink(z, out_dtype))
    return np.stack(outs)


@pytest.mark.parametrize("case,precision,out_dtype", [
    (FULL, "mixed", "f16"), (FULL, "fp32", "f16"), (FULL, "mixed", "int16"), (SMALL, "fp32", "int16"),
    (SMALL, "mixed", "int8")], ids=["full-mixed-f16", "full-fp32-f16", "full-mixed-int16", "small-fp32-int16",
                                    "small-mixed-int8"])
def test_slot_downlink_vs_oracle(case, precision, out_dtype):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import megastation_b200 as mb
    from megastation_b200 import datagen, slot
    cfg = datagen.CellConfig(**case)
    d = datagen.make_slot(cfg)
    D = 5 if cfg.M == 256 else 2
    rng = np.random.default_rng(cfg.seed + 1)
    table = datagen.mod_table(cfg.Qm)
    syms = table[rng.integers(0, 1 << cfg.Qm, (D, cfg.K, cfg.S))].astype(np.complex64)
    run = slot.UplinkSlot(cfg, precision=precision, sym_batch=cfg.U, use_graph=True, D=D, out_dtype=out_dtype)
    np_dt = {"f16": np.float16, "int16": np.int16, "int8": np.int8}[out_dtype]
    out = torch.zeros(D, cfg.M, cfg.N, 2, dtype={"f16": torch.float16, "int16": torch.int16,
                                                 "int8": torch.int8}[out_dtype], device="cuda")
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        llr, hard = run(torch.from_numpy(d["iq"]).cuda(), stream=s)
        run.downlink(torch.from_numpy(syms).cuda(), out, stream=s)
    s.synchronize()
    assert mb.ops.device_error() == 0
    assert (run.status.cpu().numpy() == 0).all()
    W, ref_up = oracle_uplink(cfg, d)
    # the uplink half of the same slot
    check_uplink(cfg, ref_up, llr.cpu().numpy(), hard.cpu().numpy(), precision, "uplink")
    ref = _downlink_ref(cfg, W, syms, np_dt).astype(np.float32)
    got = out.cpu().numpy().astype(np.float32)
    rms = np.sqrt(np.mean(ref ** 2))
    assert rms > (1.0 if out_dtype != "f16" else 1e-5)
    err = np.abs(got - ref)
    # mixed: W from BF16 operands (about 2^-9 relative); FP32: W from the
    # reference's Cholesky in FP32.  Integer outputs add one LSB of rounding.
    rel = 1e-2 if precision == "mixed" else 2e-4
    lsb = 1.0 if out_dtype in ("int16", "int8") else 0.0
    assert np.sqrt(np.mean(err ** 2)) <= rel * rms + lsb, (np.sqrt(np.mean(err ** 2)), rms)
    assert err.max() <= 8 * rel * np.abs(ref).max() + lsb + (2.0 ** -10) * np.abs(ref).max()
    # the guard bins carry nothing: each antenna row is zero outside the data band
    bins = (np.arange(cfg.S) + cfg.start + cfg.N // 2) % cfg.N
    guard = np.ones(cfg.N, bool)
    guard[bins] = False
    if out_dtype == "f16":
        spec = np.fft.fft(got[..., 0] + 1j * got[..., 1], axis=-1)
        assert np.abs(spec[..., guard]).max() <= 1e-2 * np.abs(spec[..., ~guard]).max()


def test_slot_downlink_from_bits_vs_oracle():
    # mb_slot_downlink_bits: encoded bits -> the oracle's modulation
    # (modulation.cu:115-128), precoding and inverse FFT; row length padded
    # past ceil(S Qm / 8) to check the stride
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import megastation_b200 as mb
    from megastation_b200 import datagen, slot
    cfg = datagen.CellConfig(**SMALL)
    d = datagen.make_slot(cfg)
    D = 2
    in_bytes = (cfg.S * cfg.Qm + 7) // 8 + 5
    rng = np.random.default_rng(cfg.seed + 2)
    bits = rng.integers(0, 256, (D, cfg.K, in_bytes), dtype=np.uint8)
    run = slot.UplinkSlot(cfg, precision="mixed", sym_batch=cfg.U, D=D, out_dtype="int16")
    out = torch.zeros(D, cfg.M, cfg.N, 2, dtype=torch.int16, device="cuda")
    run(torch.from_numpy(d["iq"]).cuda())
    run.downlink_bits(torch.from_numpy(bits).cuda(), out)
    torch.cuda.synchronize()
    assert mb.ops.device_error() == 0
    W, _ = oracle_uplink(cfg, d)
    syms = np.stack([orc.modulate(bits[l], cfg.S, cfg.Qm) for l in range(D)])
    ref = _downlink_ref(cfg, W, syms, np.int16).astype(np.float32)
    got = out.cpu().numpy().astype(np.float32)
    rms = np.sqrt(np.mean(ref ** 2))
    assert rms > 1.0
    # W from BF16 operands (about 2^-9 relative), one LSB of output rounding
    assert np.sqrt(np.mean((got - ref) ** 2)) <= 1e-2 * rms + 1.0
    # too short a row is refused
    from megastation_b200._lib import MbError
    with pytest.raises(MbError):
        run.downlink_bits(torch.from_numpy(bits[..., :in_bytes - 6].copy()).cuda(), out)
