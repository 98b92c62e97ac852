"""The LDPC restatement (oracle/ldpc.py) against the reference's own encoder.

The fixtures (tests/golden/ldpc/, made by tests/golden/make_ldpc_golden.py)
hold the reference's nrLDPCEncode codewords (matlab/codegen/lib/
data_generator, the generator behind the reference's test data) for seeded
information bits of base graphs 1 and 2 at Z = 16, and the parity-check
matrix of that code recovered from its outputs.  The reference itself
decodes with cuPHY, which is not in its tree: the decoder is held to round
trips here and to this restatement bit for bit on the GPU."""
import os

import numpy as np
import pytest

from oracle import ldpc

GOLD = os.path.join(os.path.dirname(__file__), "golden", "ldpc")


def _fixture(bg):
    f = np.load(os.path.join(GOLD, f"bg{bg}_z16.npz"))
    return f["entries"], f["info"], f["codewords"], int(f["Z"])


@pytest.mark.parametrize("bg", [1, 2])
def test_graph_has_the_nr_shape(bg):
    entries, _, _, Z = _fixture(bg)
    # 316 circulants in BG1, 197 in BG2 (TS 38.212 tables 5.3.2-2 and -3)
    assert len(entries) == {1: 316, 2: 197}[bg]
    kb = ldpc.KB[bg]
    for r, c, s in entries:
        assert 0 <= s < Z
        if c >= kb + 4:
            assert r >= 4 and c == kb + r and s == 0
        if r < 4:
            assert c < kb + 4


@pytest.mark.parametrize("bg", [1, 2])
def test_restated_encoder_matches_reference_codewords(bg):
    entries, info, cw, Z = _fixture(bg)
    g = ldpc.Graph(entries, ldpc.KB[bg], Z, ldpc.ROWS[bg])
    for k in range(len(info)):
        x = ldpc.encode(g, info[k])
        assert ldpc.syndrome_ok(g, x)
        np.testing.assert_array_equal(x[2 * Z:], cw[k])


@pytest.mark.parametrize("bg", [1, 2])
def test_reference_codewords_satisfy_every_parity_row(bg):
    entries, info, cw, Z = _fixture(bg)
    g = ldpc.Graph(entries, ldpc.KB[bg], Z, ldpc.ROWS[bg])
    for k in range(len(info)):
        assert ldpc.syndrome_ok(g, np.concatenate([info[k][:2 * Z], cw[k]]))


@pytest.mark.parametrize("bg,mb", [(1, 46), (1, 25), (2, 42), (2, 14)])
def test_restated_decoder_corrects_noise(bg, mb):
    entries, info, _, Z = _fixture(bg)
    g = ldpc.Graph(entries, ldpc.KB[bg], Z, mb)
    rng = np.random.default_rng(bg * 100 + mb)
    for k in range(len(info)):
        x = ldpc.encode(g, info[k])
        y = (1.0 - 2.0 * x) + 0.5 * rng.standard_normal(len(x))
        llr = (2.0 * y / 0.25).astype(np.float16)
        llr[:2 * Z] = 0  # punctured
        bits, _ = ldpc.decode(g, llr, 8)
        np.testing.assert_array_equal(bits, info[k])


def test_singular_core_is_refused():
    entries, _, _, Z = _fixture(2)
    e = entries.copy()
    # the same shift on every core parity entry of row 1 as row 0 makes rows
    # 0 and 1 equal on the core block
    core = [i for i, (r, c, s) in enumerate(e) if r < 2 and 10 <= c < 14]
    e = np.array([t for t in e if not (t[0] == 1 and 10 <= t[1] < 14)] +
                 [(1, c, s) for r, c, s in e if r == 0 and 10 <= c < 14])
    assert core
    g = ldpc.Graph(e, 10, Z, 42)
    with pytest.raises(ValueError):
        g.core_inverse()


@pytest.mark.parametrize("bg", [1, 2])
def test_restated_decoder_bounds(bg):
    """The float16 decoder's bounds (channel LLRs clamped to +-1024, messages
    to +-256, q and app unclamped sums) keep every value finite over the
    32 passes allowed, from LLRs at the FP16 limit and infinities, and the
    confident codewords decode; more passes are refused."""
    entries, info, _, Z = _fixture(bg)
    g = ldpc.Graph(entries, ldpc.KB[bg], Z, ldpc.ROWS[bg])
    for k in range(2):
        x = ldpc.encode(g, info[k])
        llr = np.clip((1.0 - 2.0 * x) * 65504.0, -65504, 65504).astype(np.float16)
        llr[2 * Z + k] = np.inf if llr[2 * Z + k] > 0 else -np.inf
        bits, app = ldpc.decode(g, llr, ldpc.MAX_ITER)
        assert np.isfinite(app.astype(np.float32)).all()
        assert np.abs(app.astype(np.float32)).max() <= 1024 + ldpc.ROWS[bg] * 256 + 2048
        np.testing.assert_array_equal(bits, info[k])
    with pytest.raises(AssertionError):
        ldpc.decode(g, llr, ldpc.MAX_ITER + 1)
