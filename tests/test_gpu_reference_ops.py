"""The uplink slot against the reference's own CUDA operators (cuFFT,
cuBLAS/cuSOLVER, the SIMT equalizer), built from the reference tree into
oracle/_ref: LLRs of the plain and mixed paths on int16 samples, with the
tolerances of the oracle tests.  Skipped where the reference library was not
built."""
import numpy as np
import pytest
import torch

from oracle import ref_ops

pytestmark = pytest.mark.gpu


@pytest.mark.skipif(not ref_ops.available(), reason="oracle/_ref/libref_ops.so not built")
@pytest.mark.parametrize("iq_dtype", ["int16", "int8"])
@pytest.mark.parametrize("precision", ["fp32", "mixed"])
def test_slot_matches_reference_operators(precision, iq_dtype):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from megastation_b200 import datagen, slot
    cfg = datagen.CellConfig(M=64, K=16, N=2048, S=1200, sg=16, Qm=4, U=4, snr_db=25.0, iq_dtype=iq_dtype,
                             seed=21)
    d = datagen.make_slot(cfg)
    cb, zeros, stride = cfg.ldpc()
    iq = torch.from_numpy(d["iq"]).cuda()
    stream = torch.cuda.Stream()
    ref = ref_ops.RefSlot(cfg.M, cfg.K, cfg.N, cfg.S, cfg.sg, cfg.Qm, cfg.P, cfg.U, cb, zeros, stride,
                          iq=iq_dtype)
    llr_ref = torch.zeros(cfg.U, cfg.K, stride, dtype=torch.float16, device="cuda")
    ref.uplink(iq.data_ptr(), llr_ref.data_ptr(), stream.cuda_stream)
    run = slot.UplinkSlot(cfg, precision=precision, sym_batch=cfg.U)
    with torch.cuda.stream(stream):
        llr, _ = run(iq, stream=stream)
    stream.synchronize()
    a = llr.cpu().numpy().astype(np.float32)
    r = llr_ref.cpu().numpy().astype(np.float32)
    n_valid = min(cb, cfg.S * cfg.Qm)
    a, r = a[..., zeros:zeros + n_valid], r[..., zeros:zeros + n_valid]
    sure = np.abs(r) > 4.0
    assert sure.mean() > 0.5
    assert ((a[sure] < 0) == (r[sure] < 0)).all()
    tol = 0.25 if precision == "fp32" else 1.0
    assert np.abs(a - r).max() <= tol + 0.02 * np.abs(r).max(), np.abs(a - r).max()


@pytest.mark.skipif(not ref_ops.available(), reason="oracle/_ref/libref_ops.so not built")
@pytest.mark.parametrize("precision", ["fp32", "mixed"])
def test_bench_slot_int8_matches_reference_operators(precision):
    """The bench's slot (256x32, N = 4096, S = 3276, 12 uplink symbols) on
    int8 samples, the reference's production format: the mixed path runs the
    tensor-core FFT here.  The reference beamforms whole groups only
    (S / sg = 204 of them), so the last, partial group's subcarriers
    (3264..3275) are left out of the comparison."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from megastation_b200 import datagen, slot
    cfg = datagen.CellConfig(M=256, K=32, N=4096, S=3276, sg=16, Qm=6, U=12, snr_db=25.0, channel="tdl",
                             n_taps=8, tap_decay=2.0, rho=0.5, iq_dtype="int8", seed=23)
    d = datagen.make_slot(cfg)
    cb, zeros, stride = cfg.ldpc()
    iq = torch.from_numpy(d["iq"]).cuda()
    stream = torch.cuda.Stream()
    ref = ref_ops.RefSlot(cfg.M, cfg.K, cfg.N, cfg.S, cfg.sg, cfg.Qm, cfg.P, cfg.U, cb, zeros, stride,
                          iq="int8")
    llr_ref = torch.zeros(cfg.U, cfg.K, stride, dtype=torch.float16, device="cuda")
    ref.uplink(iq.data_ptr(), llr_ref.data_ptr(), stream.cuda_stream)
    run = slot.UplinkSlot(cfg, precision=precision, sym_batch=cfg.U)
    with torch.cuda.stream(stream):
        llr, _ = run(iq, stream=stream)
    stream.synchronize()
    a = llr.cpu().numpy().astype(np.float32)
    r = llr_ref.cpu().numpy().astype(np.float32)
    n_whole = min(cb, (cfg.S // cfg.sg) * cfg.sg * cfg.Qm)
    a, r = a[..., zeros:zeros + n_whole], r[..., zeros:zeros + n_whole]
    sure = np.abs(r) > 4.0
    assert sure.mean() > 0.5
    assert ((a[sure] < 0) == (r[sure] < 0)).all()
    tol = 0.25 if precision == "fp32" else 1.0
    assert np.abs(a - r).max() <= tol + 0.02 * np.abs(r).max(), np.abs(a - r).max()
