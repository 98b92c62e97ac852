"""The LDPC kernels (csrc/ldpc.cu through the C ABI) against the reference's
encoder and the float16 restatement of the decoder (oracle/ldpc.py).

The encoder must give the reference's nrLDPCEncode codewords bit for bit
(tests/golden/ldpc/, base graphs 1 and 2 at Z = 16) and the restated encoder's
on fewer parity rows and on a Z = 384 graph of base graph 1's shape; the
decoder must give the restatement's information bits bit for bit on noisy
FP16 LLRs, including where it fails to correct, for odd batches (a pair's
second block absent) and for LLRs at the FP16 limit (the a-posteriori clamp),
and recover the information of moderately noisy codewords."""
import os

import numpy as np
import pytest
import torch

from oracle import ldpc

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden", "ldpc")


def _fixture(bg):
    f = np.load(os.path.join(GOLD, f"bg{bg}_z16.npz"))
    return f["entries"], f["info"], f["codewords"], int(f["Z"])


def _big_graph(Z=384, seed=0):
    """Base graph 1's circulant pattern with seeded shifts at Z = 384 (an
    invertible core block), for production-size kernels."""
    entries, _, _, _ = _fixture(1)
    rng = np.random.default_rng(seed)
    while True:
        e = entries.copy()
        kb = ldpc.KB[1]
        for k, (r, c, s) in enumerate(e):
            e[k, 2] = 0 if c >= kb + 4 else rng.integers(0, Z)
        try:
            ldpc.Graph(e, kb, Z, 4).core_inverse()
            return e
        except ValueError:
            continue


def _mb():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import megastation_b200 as mb
    return mb


def _pack(bits):
    return torch.from_numpy(np.packbits(bits, axis=-1)).cuda()


@pytest.mark.parametrize("bg", [1, 2])
def test_encoder_matches_reference_codewords(bg):
    mb = _mb()
    entries, info, cw, Z = _fixture(bg)
    code = mb.Ldpc(entries, ldpc.KB[bg], Z, ldpc.ROWS[bg])
    out = code.encode(_pack(info))
    torch.cuda.synchronize()
    got = np.unpackbits(out.cpu().numpy(), axis=1)[:, :cw.shape[1]]
    np.testing.assert_array_equal(got, cw)


@pytest.mark.parametrize("case", ["bg1-z16-mb25", "bg2-z16-mb14", "bg1-z384-mb46", "bg1-z384-mb12"])
def test_encoder_matches_restatement(case):
    mb = _mb()
    bg = 2 if case.startswith("bg2") else 1
    Z = int(case.split("-")[1][1:])
    m = int(case.split("-")[2][2:])
    entries = _fixture(bg)[0] if Z == 16 else _big_graph(Z)
    kb = ldpc.KB[bg]
    g = ldpc.Graph(entries, kb, Z, m)
    rng = np.random.default_rng(Z + m)
    info = rng.integers(0, 2, (5, kb * Z), dtype=np.uint8)
    code = mb.Ldpc(entries, kb, Z, m)
    # a padded output row: the stride is the caller's
    out = torch.zeros(5, (code.cw_bits + 7) // 8 + 3, dtype=torch.uint8, device="cuda")
    code.encode(_pack(info), out=out)
    torch.cuda.synchronize()
    got = np.unpackbits(out.cpu().numpy(), axis=1)[:, :code.cw_bits]
    for k in range(5):
        np.testing.assert_array_equal(got[k], ldpc.encode(g, info[k])[2 * Z:])


@pytest.mark.parametrize("case", ["bg1-z16-mb46", "bg2-z16-mb42", "bg2-z16-mb14", "bg1-z384-mb46"])
@pytest.mark.parametrize("sigma,iters", [(0.5, 8), (0.9, 3), (1.3, 5)])
def test_decoder_matches_restatement(case, sigma, iters):
    mb = _mb()
    bg = 2 if case.startswith("bg2") else 1
    Z = int(case.split("-")[1][1:])
    m = int(case.split("-")[2][2:])
    entries = _fixture(bg)[0] if Z == 16 else _big_graph(Z)
    kb = ldpc.KB[bg]
    g = ldpc.Graph(entries, kb, Z, m)
    B = 7 if Z == 16 else 3  # odd: the last pair has one block
    rng = np.random.default_rng(int(sigma * 100) + Z + m)
    info = rng.integers(0, 2, (B, kb * Z), dtype=np.uint8)
    # equalizer-style rows: the code block's LLRs, punctured ones zero, then
    # unused tail up to the row stride
    stride = g.N + 24
    llr = np.zeros((B, stride), np.float16)
    for k in range(B):
        x = ldpc.encode(g, info[k])
        y = (1.0 - 2.0 * x) + sigma * rng.standard_normal(len(x))
        llr[k, :g.N] = (2.0 * y / sigma ** 2).astype(np.float16)
        llr[k, :2 * Z] = 0
    code = mb.Ldpc(entries, kb, Z, m, max_batch=4)  # B = 7 decodes in two turns
    out = code.decode(torch.from_numpy(llr).cuda(), max_iter=iters)
    torch.cuda.synchronize()
    assert mb.ops.device_error() == 0
    got = np.unpackbits(out.cpu().numpy(), axis=1)[:, :kb * Z]
    decoded = 0
    for k in range(B):
        bits, _ = ldpc.decode(g, llr[k, :g.N], iters)
        np.testing.assert_array_equal(got[k], bits, err_msg=f"block {k}")
        decoded += int((bits == info[k]).all())
    if sigma <= 0.5:
        assert decoded == B


@pytest.mark.parametrize("bg", [1, 2])
def test_decoder_clamps_large_llrs(bg):
    """LLRs up to the FP16 limit (and infinities), 32 passes: channel LLRs
    clamped to +-1024 and messages to +-256 keep every value finite, the
    kernel equals the restatement, bounds included, bit for bit, and the
    confident codewords decode; more than 32 passes are refused."""
    mb = _mb()
    entries, info, _, Z = _fixture(bg)
    kb = ldpc.KB[bg]
    g = ldpc.Graph(entries, kb, Z, ldpc.ROWS[bg])
    rng = np.random.default_rng(40 + bg)
    B = 3
    llr = np.zeros((B, g.N), np.float16)
    for k in range(B):
        x = ldpc.encode(g, info[k])
        y = (1.0 - 2.0 * x) * rng.uniform(2e3, 7e4, len(x))
        y[rng.integers(0, len(x), 8)] *= -1  # a few confident errors
        llr[k] = np.clip(y, -65504, 65504).astype(np.float16)
        llr[k, :2 * Z] = 0
    llr[0, 2 * Z + 5] = np.inf
    llr[1, 2 * Z + 9] = -np.inf
    llr[2, 2 * Z + 3] = np.float16(-0.0)  # a negative zero counts as negative
    code = mb.Ldpc(entries, kb, Z, ldpc.ROWS[bg], max_batch=B)
    out = code.decode(torch.from_numpy(llr).cuda(), max_iter=32)
    torch.cuda.synchronize()
    got = np.unpackbits(out.cpu().numpy(), axis=1)[:, :kb * Z]
    bits, app = ldpc.decode(g, llr, 32)
    assert np.isfinite(app.astype(np.float32)).all()
    np.testing.assert_array_equal(got, bits)
    np.testing.assert_array_equal(bits, info[:B])
    from megastation_b200._lib import MbError
    with pytest.raises(MbError):
        code.decode(torch.from_numpy(llr).cuda(), max_iter=33)


def test_graph_errors():
    mb = _mb()
    from megastation_b200._lib import MbError
    entries, _, _, Z = _fixture(2)
    bad = entries.copy()
    bad[-1, 1] = 200  # a column past the graph
    with pytest.raises(MbError):
        mb.Ldpc(bad, 10, Z, 42)
    with pytest.raises(MbError):
        mb.Ldpc(entries, 10, Z, 3)  # fewer than the four core rows


@pytest.mark.parametrize("precision", ["mixed", "fp32"])
def test_slot_uplink_decodes_the_reference_code(precision):
    """The reference's uplink order end to end (process.cc:161-189): a cell
    whose code block is base graph 1 at Z = 16 (S Qm = 1056 coded bits per
    (symbol, user), the config.cc sizing at rate 1/3); information bits
    scrambled by the LFSR sequence and encoded as the reference's encoder
    does, sent over the channel; the slot's LLRs through mb_slot_decode
    (LDPC decode, then descramble) give the information bits back."""
    mb = _mb()
    from oracle import oracle as orc

    from megastation_b200 import datagen, slot
    cfg = datagen.CellConfig(M=16, K=4, N=512, S=264, sg=8, Qm=4, U=2, snr_db=20.0, seed=71)
    cb, zeros, stride = cfg.ldpc()
    entries, _, _, Z = _fixture(1)
    kb, m = ldpc.KB[1], ldpc.ROWS[1]
    assert (cb, zeros) == ((kb - 2 + m) * Z, 2 * Z)
    g = ldpc.Graph(entries, kb, Z, m)
    rng = np.random.default_rng(72)
    info = rng.integers(0, 2, (cfg.U, cfg.K, kb * Z), dtype=np.uint8)
    seq = orc.scrambler_seq127()
    scrambled = info ^ seq[np.arange(kb * Z) % 127]
    coded = np.stack([np.stack([ldpc.encode(g, scrambled[l, u])[2 * Z:] for u in range(cfg.K)])
                      for l in range(cfg.U)])
    d = datagen.make_slot(cfg, coded=coded)
    run = slot.UplinkSlot(cfg, precision=precision, sym_batch=cfg.U)
    code = mb.Ldpc(entries, kb, Z, m)
    run.set_ldpc(code, max_iter=8)
    llr, _ = run(torch.from_numpy(d["iq"]).cuda())
    out = run.decode(llr)
    torch.cuda.synchronize()
    assert mb.ops.device_error() == 0
    got = np.unpackbits(out.cpu().numpy(), axis=-1)[..., :kb * Z]
    np.testing.assert_array_equal(got, info)
    # a code that does not fit the cell's LLR layout is refused
    from megastation_b200._lib import MbError
    with pytest.raises(MbError):
        run.set_ldpc(mb.Ldpc(entries, kb, Z, 20))


def test_slot_downlink_from_information_bits():
    """process.cc:196-214 from information bits (mb_slot_downlink_info):
    the same antenna samples as the downlink of the LFSR-scrambled bits
    encoded by the reference's encoder (the restatement, pinned to it above)
    through mb_slot_downlink_bits."""
    mb = _mb()
    from oracle import oracle as orc

    from megastation_b200 import datagen, slot
    cfg = datagen.CellConfig(M=16, K=4, N=512, S=264, sg=8, Qm=4, U=2, snr_db=20.0, seed=73)
    entries, _, _, Z = _fixture(1)
    kb, m = ldpc.KB[1], ldpc.ROWS[1]
    g = ldpc.Graph(entries, kb, Z, m)
    D = 2
    rng = np.random.default_rng(74)
    info = rng.integers(0, 2, (D, cfg.K, kb * Z), dtype=np.uint8)
    seq = orc.scrambler_seq127()
    coded = np.stack([np.stack([ldpc.encode(g, info[l, u] ^ seq[np.arange(kb * Z) % 127])[2 * Z:]
                                for u in range(cfg.K)]) for l in range(D)])
    d = datagen.make_slot(cfg)
    run = slot.UplinkSlot(cfg, precision="mixed", sym_batch=cfg.U, D=D, out_dtype="int16")
    run.set_ldpc(mb.Ldpc(entries, kb, Z, m))
    run(torch.from_numpy(d["iq"]).cuda())
    a = torch.zeros(D, cfg.M, cfg.N, 2, dtype=torch.int16, device="cuda")
    b = torch.zeros_like(a)
    run.downlink_info(_pack(info), a)
    run.downlink_bits(_pack(coded), b)
    torch.cuda.synchronize()
    assert mb.ops.device_error() == 0
    assert a.abs().max().item() > 0
    assert torch.equal(a, b)
