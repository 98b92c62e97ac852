"""Batched uneven cells (one CUDA graph launch per slot) against the same
cells run one at a time through the single-cell slot runner: the kernels and
inputs are the same, so LLRs and hard bits must match bit for bit, before and
after the autotuner changes the batching, the equalizer tiles and the FFT's
CTAs; and every cell against the FP64 oracle, whichever product path the
mixed ZF takes."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cells_data():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from megastation_b200 import datagen
    cfgs = datagen.make_cells(n=6, seed=11)
    slots = [datagen.make_slot(c) for c in cfgs]
    iqs = [torch.from_numpy(s["iq"]).cuda() for s in slots]
    return cfgs, iqs


def _single(cfg, iq, precision):
    from megastation_b200 import slot
    run = slot.UplinkSlot(cfg, precision=precision, sym_batch=max(cfg.U, 1))
    llr, hard = run(iq)
    torch.cuda.synchronize()
    return llr.cpu().numpy().view(np.uint16), hard.cpu().numpy(), run.status.cpu().numpy()


@pytest.mark.parametrize("precision", ["mixed", "fp32"])
def test_cells_match_single_cell_slots(cells_data, precision):
    from megastation_b200 import cells
    cfgs, iqs = cells_data
    cs = cells.Cells(cfgs, precision=precision)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        cs(iqs, stream=s)
        llr, hard = cs(iqs, stream=s)  # replay of the captured graph
    s.synchronize()
    for c, cfg in enumerate(cfgs):
        l1, h1, st1 = _single(cfg, iqs[c], precision)
        np.testing.assert_array_equal(llr[c].cpu().numpy().view(np.uint16), l1, err_msg=f"cell {c}")
        np.testing.assert_array_equal(hard[c].cpu().numpy(), h1, err_msg=f"cell {c}")
        np.testing.assert_array_equal(cs.status[c].cpu().numpy(), st1)


def test_cells_autotune_keeps_results(cells_data):
    from megastation_b200 import cells
    cfgs, iqs = cells_data
    cs = cells.Cells(cfgs, precision="mixed")
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        ref_llr, ref_hard = cs(iqs, stream=s)
        ref = [(a.clone(), b.clone()) for a, b in zip(ref_llr, ref_hard)]
        choice, us = cs.autotune(iqs, reps=5, stream=s)
    s.synchronize()
    assert us > 0
    assert cs.tuning() == choice
    # the ZF's product path changes its arithmetic; with the rule's path the
    # tuned batching, equalizer tiles and FFT CTAs give the same bits
    cs.set_tuning([{**t, "zf_path": 0} for t in choice])
    with torch.cuda.stream(s):
        llr, hard = cs(iqs, stream=s)
    s.synchronize()
    for c, cfg in enumerate(cfgs):
        assert 1 <= choice[c]["sym_batch"] <= max(cfg.U, 1)
        assert choice[c]["eq_cols"] in (64, 128)
        assert choice[c]["fft_ctas"] in (0, 74, 37, 18)
        assert choice[c]["zf_path"] in (0, 1, 2)
        assert torch.equal(llr[c], ref[c][0]) and torch.equal(hard[c], ref[c][1]), c
    # a hand-set tuning (smallest batches, narrow tiles, tensor-core FFTs on
    # 18 CTAs) gives the same bits
    cs.set_tuning([{"sym_batch": 1, "eq_cols": 64, "fft_ctas": 18} for _ in cfgs])
    assert all(t["fft_ctas"] == 18 for t in cs.tuning())
    with torch.cuda.stream(s):
        llr, hard = cs(iqs, stream=s)
    s.synchronize()
    for c in range(len(cfgs)):
        assert torch.equal(llr[c], ref[c][0]) and torch.equal(hard[c], ref[c][1]), c


@pytest.mark.parametrize("n,seed,precision,zf_path", [(32, 3, "mixed", 0), (32, 3, "mixed", 1), (32, 3, "mixed", 2),
                                                      (6, 11, "fp32", 0)],
                         ids=["bench-32-cells-mixed", "bench-32-cells-mixed-cuda-core-zf",
                              "bench-32-cells-mixed-tensor-core-zf", "6-cells-fp32"])
def test_cells_vs_oracle(n, seed, precision, zf_path):
    """Every cell of a batched slot against the FP64 oracle run on that cell
    alone (pilot FFT, ZF, FFT, equalize, descrambled hard bits); the 32-cell
    set is the batched-cells workload of the bench (seed 3), also with the
    mixed ZF's products forced onto the CUDA cores (1) or the tensor cores
    (2) for every cell with K <= 32."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import megastation_b200 as mb
    from megastation_b200 import cells, datagen

    from slot_oracle import check_uplink, oracle_uplink
    cfgs = datagen.make_cells(n=n, seed=seed)
    data = [datagen.make_slot(c) for c in cfgs]
    iqs = [torch.from_numpy(d["iq"]).cuda() for d in data]
    cs = cells.Cells(cfgs, precision=precision)
    if zf_path:
        cs.set_tuning([{**t, "zf_path": zf_path} for t in cs.tuning()])
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        cs(iqs, stream=s)
        llr, hard = cs(iqs, stream=s)
    s.synchronize()
    assert mb.ops.device_error() == 0
    for c, (cfg, d) in enumerate(zip(cfgs, data)):
        # 0: solved, 2: solved on the FP64 fallback (cells with as many users
        # as antennas have ill-conditioned groups); never 1 (not PD)
        assert np.isin(cs.status[c].cpu().numpy(), (0, 2)).all(), c
        _, ref = oracle_uplink(cfg, d)
        check_uplink(cfg, ref, llr[c].cpu().numpy(), hard[c].cpu().numpy(), precision, f"cell {c}",
                     sent=d["bits"])
