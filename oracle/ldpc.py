"""CPU restatement of the NR LDPC encode / decode around the slot (test
infrastructure, never on the product path).

The reference takes LDPC from cuPHY (operators/ldpc/encoder.h:48-75,
decoder.h:60-86), which is not in its tree; its MATLAB-generated data
generator (matlab/codegen/lib/data_generator, nrLDPCEncode) is, and
oracle/ref_ldpc.mk builds it here.  This module

* wraps that reference encoder (`ref_encode`, this container only: it needs
  oracle/_ref/libref_ldpc.so built from the reference tree);
* recovers the quasi-cyclic parity-check matrix of its code for one lifting
  size from the encoder's outputs alone (`derive_graph`): codewords of the
  unit information vectors, with the block structure every NR base graph has
  (TS 38.212 5.3.2: four core rows over the information and four core parity
  columns, then one row per extension parity column, which it carries as an
  identity block);
* restates the encoder for such a graph (`encode`: core parity from the
  inverse of the 4Z x 4Z core block, extension parity row by row) and a
  layered normalized min-sum decoder (`decode`) in the float16 arithmetic of
  the library's kernel (the precision of the reference's cuPHY decoder), for
  bit-exact comparisons.

Block (i, j) of the graph with shift s is the Z x Z identity with its
columns cyclically shifted right by s: row r has its one in column
(r + s) mod Z (TS 38.212 5.3.2).  Bits are 0/1 uint8 arrays.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(_HERE, "_ref", "libref_ldpc.so")

KB = {1: 22, 2: 10}        # information block columns
COLS = {1: 68, 2: 52}      # block columns of the full base graph
ROWS = {1: 46, 2: 42}      # block rows


# ------------------------------------------------------------ reference
class _Emx(ctypes.Structure):
    # emxArray_real_T of the generated code (data_generator_types.h:100-106)
    _fields_ = [("data", ctypes.POINTER(ctypes.c_double)), ("size", ctypes.POINTER(ctypes.c_int)),
                ("allocatedSize", ctypes.c_int), ("numDimensions", ctypes.c_int),
                ("canFreeData", ctypes.c_ubyte)]


_ref = None


def ref_available():
    return os.path.exists(REF_LIB)


def _ref_lib():
    global _ref
    if _ref is None:
        _ref = ctypes.CDLL(REF_LIB)
        _ref.data_generator_initialize()
        _ref.nrLDPCEncode.argtypes = [ctypes.POINTER(_Emx), ctypes.c_double, ctypes.POINTER(_Emx)]
        _ref.nrLDPCEncode.restype = None
    return _ref


def ref_encode(info, bgn):
    """The reference's nrLDPCEncode on info [C][kb Z] (0/1): codewords
    [C][(cols - 2) Z], the first 2Z systematic bits punctured."""
    lib = _ref_lib()
    info = np.asarray(info, dtype=np.float64)
    C, K = info.shape
    col_major = np.ascontiguousarray(info)  # a K x C column-major array is [C][K] in C order
    ins = (ctypes.c_int * 2)(K, C)
    a = _Emx(col_major.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), ins, K * C, 2, 0)
    outs = (ctypes.c_int * 2)(0, 0)
    b = _Emx(None, outs, 0, 2, 1)
    lib.nrLDPCEncode(ctypes.byref(a), float(bgn), ctypes.byref(b))
    N, C2 = outs[0], outs[1]
    out = np.ctypeslib.as_array(b.data, shape=(C2 * N,)).copy()
    return np.rint(out.reshape(C2, N)).astype(np.uint8)


# --------------------------------------------------------------- graphs
def _shift(v, s):
    """(P^s v)[r] = v[(r + s) mod Z] for v [..., Z]."""
    return np.roll(v, -s, axis=-1)


def derive_graph(bgn, Z):
    """Block entries (row, col, shift) of the parity-check matrix of the
    reference encoder's code at lifting size Z, from its codewords alone.
    For block row i, the unit information vector of block j0 (bit 0) gives
    sum over the row's core parity columns m of P^s_im p_m + (extension
    row: its own parity block) = the row's j0 term, which is zero or one
    bit at (-s_i,j0) mod Z; the core columns' shifts are found by search (at
    most four of them, Z + 1 choices each; of several consistent rows the
    sparsest), the information shifts read off.  Exhaustive in Z^3: meant
    for small Z."""
    kb, cols, rows = KB[bgn], COLS[bgn], ROWS[bgn]
    info = np.zeros((kb, kb * Z), np.uint8)
    for j in range(kb):
        info[j, j * Z] = 1
    cw = ref_encode(info, bgn)                                     # [kb][(cols - 2) Z]
    x = np.concatenate([info[:, :2 * Z], cw], axis=1).reshape(kb, cols, Z)  # full codewords
    core = [x[:, kb + m, :] for m in range(4)]                     # [kb][Z] each
    shifted = np.stack([np.stack([_shift(core[m], s) for s in range(Z)]) for m in range(4)])  # [4][Z][kb][Z]
    opts = [None] + list(range(Z))

    def search(own, core_row):
        """Every (weight, core shifts, per-j0 residual) consistent with own."""
        out = []
        for s0 in opts:
            a0 = own ^ (shifted[0, s0] if s0 is not None else 0)
            for s1 in opts:
                a1 = a0 ^ (shifted[1, s1] if s1 is not None else 0)
                for s2 in opts:
                    a2 = a1 ^ (shifted[2, s2] if s2 is not None else 0)
                    # the last column vectorised over its Z + 1 choices
                    cand = np.concatenate([a2[None], a2[None] ^ shifted[3]], axis=0)  # [Z + 1][kb][Z]
                    ok = (cand.sum(axis=2) <= 1).all(axis=1)
                    for k in np.nonzero(ok)[0]:
                        sel = (s0, s1, s2, None if k == 0 else int(k - 1))
                        n_core = sum(v is not None for v in sel)
                        if core_row and n_core < 2:
                            continue  # a core row spans at least two core parity columns
                        out.append((int(cand[k].sum()) + n_core, sel, cand[k].copy()))
        out.sort(key=lambda t: t[0])
        return out

    def row_entries(i, sel, lhs):
        ents = []
        for j0 in range(kb):
            nz = np.nonzero(lhs[j0])[0]
            if len(nz):
                ents.append((i, j0, int((-nz[0]) % Z)))
        for m, sm in enumerate(sel):
            if sm is not None:
                ents.append((i, kb + m, int(sm)))
        return ents

    def core_block(sel):
        # the candidate's Z bit rows on the core parity columns
        B = np.zeros((Z, 4 * Z), np.uint8)
        for m, sm in enumerate(sel):
            if sm is not None:
                for r in range(Z):
                    B[r, m * Z + (r + sm) % Z] ^= 1
        return B

    def rank2(M):
        M = M.copy()
        r = 0
        for c in range(M.shape[1]):
            piv = np.nonzero(M[r:, c])[0]
            if len(piv) == 0:
                continue
            p = r + piv[0]
            M[[r, p]] = M[[p, r]]
            others = np.nonzero(M[:, c])[0]
            M[others[others != r]] ^= M[r]
            r += 1
            if r == M.shape[0]:
                break
        return r

    # the core rows span every valid row over the information and core parity
    # columns only: take the sparsest four whose core blocks are independent
    entries = []
    chosen = np.zeros((0, 4 * Z), np.uint8)
    for w, sel, lhs in search(np.zeros((kb, Z), np.uint8), True):
        B = np.concatenate([chosen, core_block(sel)])
        if rank2(B) == B.shape[0]:
            entries += row_entries(len(chosen) // Z, sel, lhs)
            chosen = B
            if len(chosen) == 4 * Z:
                break
    if len(chosen) != 4 * Z:
        raise ValueError("no four independent core rows")
    # each extension row: its own parity block plus the sparsest consistent rest
    for i in range(4, rows):
        found = search(x[:, kb + i, :], False)
        if not found:
            raise ValueError(f"row {i}: no consistent core columns")
        _, sel, lhs = found[0]
        entries += row_entries(i, sel, lhs)
        entries.append((i, kb + i, 0))
    return np.array(sorted(entries), dtype=np.int32)


class Graph:
    """A base graph (entries [n][3] of (row, col, shift)) at lifting Z, of
    which the first mb block rows are used (mb = parity nodes: code rate)."""

    def __init__(self, entries, kb, Z, mb):
        self.entries = np.asarray(entries, dtype=np.int64)
        self.kb, self.Z, self.mb = kb, Z, mb
        self.rows = [[(int(c), int(s)) for r, c, s in self.entries if r == i] for i in range(mb)]
        self.N = (kb + mb) * Z
        self._binv = None

    def core_inverse(self):
        """B^-1 over GF(2), B the 4Z x 4Z block of the core rows on the core
        parity columns: B[(i, r), (m, (r + s) mod Z)] = 1."""
        if self._binv is None:
            Z, kb = self.Z, self.kb
            B = np.zeros((4 * Z, 4 * Z), np.uint8)
            for i in range(4):
                for c, s in self.rows[i]:
                    if kb <= c < kb + 4:
                        for r in range(Z):
                            B[i * Z + r, (c - kb) * Z + (r + s) % Z] ^= 1
            n = 4 * Z
            aug = np.concatenate([B, np.eye(n, dtype=np.uint8)], axis=1)
            for col in range(n):
                piv = col + np.nonzero(aug[col:, col])[0]
                if len(piv) == 0:
                    raise ValueError("singular core block")
                p = piv[0]
                if p != col:
                    aug[[col, p]] = aug[[p, col]]
                rows = np.nonzero(aug[:, col])[0]
                rows = rows[rows != col]
                aug[rows] ^= aug[col]
            self._binv = aug[:, n:].copy()
        return self._binv


def encode(g, info):
    """Full codeword [(kb + mb) Z] (punctured systematic bits included) of
    info [kb Z]: core parity B^-1 A s, then each extension row's parity."""
    Z, kb = g.Z, g.kb
    x = np.zeros((kb + g.mb, Z), np.uint8)
    x[:kb] = np.asarray(info, np.uint8).reshape(kb, Z)
    lam = np.zeros((4, Z), np.uint8)
    for i in range(4):
        for c, s in g.rows[i]:
            if c < kb:
                lam[i] ^= _shift(x[c], s)
    p = (g.core_inverse().astype(np.int64) @ lam.reshape(-1).astype(np.int64)) & 1
    x[kb:kb + 4] = p.reshape(4, Z).astype(np.uint8)
    for i in range(4, g.mb):
        acc = np.zeros(Z, np.uint8)
        for c, s in g.rows[i]:
            if c != kb + i:
                acc ^= _shift(x[c], s)
        x[kb + i] = acc
    return x.reshape(-1)


def syndrome_ok(g, x):
    Z = g.Z
    xb = np.asarray(x, np.uint8).reshape(-1, Z)
    for i in range(g.mb):
        acc = np.zeros(Z, np.uint8)
        for c, s in g.rows[i]:
            acc ^= _shift(xb[c], s)
        if acc.any():
            return False
    return True


# FP16 range: the channel LLRs are clamped to +-LLR_MAX once and every
# check-to-variable message to +-MSG_MAX, while q and app are exact sums
# (app = llr + the sum of the messages of its rows, up to rounding); with
# at most 46 rows a variable stays below 1024 + 46 * 256 = 12800, and the
# rounding of two operations a row visit (at most 32 below 65504) adds at
# most 46 * 32 * 32 over 32 passes: nothing overflows for max_iter <= 32
LLR_MAX = np.float16(1024)
MSG_MAX = np.float16(256)
MAX_ITER = 32


def decode(g, llr, max_iter, alpha=0.75):
    """Layered normalized min-sum over the first mb block rows, rows in
    order, max_iter passes, float16 arithmetic in the library kernel's order
    (every step one IEEE float16 operation, round to nearest even):
    app = clip(llr, +-LLR_MAX); per row, for each check node q = app - c2v,
    min1 = min |q| (first index), min2 = the least of the others (min1 for a
    single entry), the parity of the sign bits of q (-0 counts as negative);
    r = +-min(alpha * min, MSG_MAX)
    (alpha * min2 at min1's index); app = q + r.  llr [(kb + mb) Z]
    (float16; positive means bit 0), or [B][(kb + mb) Z] for B independent
    blocks.  Returns (bits [kb Z] or [B][kb Z], app)."""
    Z, kb = g.Z, g.kb
    x = np.asarray(llr, np.float16)
    one = x.ndim == 1
    assert max_iter <= MAX_ITER
    app = np.clip(np.atleast_2d(x), -LLR_MAX, LLR_MAX).T.copy()       # [N][B]
    a = np.float16(alpha)
    z = np.arange(Z)
    idx = [np.stack([c * Z + (z + s) % Z for c, s in ents]) for ents in g.rows]
    B = app.shape[1]
    c2v = [np.zeros((len(ents), Z, B), np.float16) for ents in g.rows]
    for _ in range(max_iter):
        for i in range(g.mb):
            q = app[idx[i]] - c2v[i]                                   # [deg][Z][B]
            mag = np.abs(q)
            deg = mag.shape[0]
            pos = np.argmin(mag, axis=0)                               # [Z][B]
            min1 = np.take_along_axis(mag, pos[None], axis=0)[0]
            if deg > 1:
                rest = mag.copy()
                np.put_along_axis(rest, pos[None], np.float16(np.inf), axis=0)
                min2 = rest.min(axis=0)
            else:
                min2 = min1
            neg = np.signbit(q)
            par = np.logical_xor.reduce(neg, axis=0)
            m1, m2 = np.minimum(a * min1, MSG_MAX), np.minimum(a * min2, MSG_MAX)
            m = np.where(np.arange(deg)[:, None, None] == pos[None], m2[None], m1[None])
            r = np.where(par[None] ^ neg, -m, m)
            app[idx[i]] = q + r
            c2v[i] = r
    bits = (app[:kb * Z] < 0).astype(np.uint8).T
    return (bits[0], app[:, 0]) if one else (bits, app.T)
