"""LDPC fixtures from the reference's own encoder, so that the LDPC parity
tests run where the reference tree is not mounted.

The reference takes LDPC from cuPHY (not in its tree); its MATLAB-generated
data generator (matlab/codegen/lib/data_generator, nrLDPCEncode) is, built
in place by oracle/ref_ldpc.mk.  For base graphs 1 and 2 at lifting size
Z = 16 this script writes tests/golden/ldpc/bg{1,2}_z16.npz with

  entries   [n][3] (row, col, shift): the parity-check matrix of that
            encoder's code, recovered from its outputs by
            oracle.ldpc.derive_graph (codewords of the unit information
            vectors; nothing is read from the reference's sources);
  info      [4][kb Z] seeded information bits;
  codewords [4][(cols - 2) Z] the reference encoder's output for them.

Usage: python tests/golden/make_ldpc_golden.py  (after
`make -C oracle -f ref_ldpc.mk REF=<MegaStation tree>`)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import ldpc  # noqa: E402

Z = 16


def main():
    if not ldpc.ref_available():
        sys.exit("oracle/_ref/libref_ldpc.so is missing: make -C oracle -f ref_ldpc.mk REF=<MegaStation tree>")
    out_dir = os.path.join(HERE, "ldpc")
    os.makedirs(out_dir, exist_ok=True)
    for bg in (1, 2):
        entries = ldpc.derive_graph(bg, Z)
        kb = ldpc.KB[bg]
        rng = np.random.default_rng(100 + bg)
        info = rng.integers(0, 2, (4, kb * Z), dtype=np.uint8)
        cw = ldpc.ref_encode(info, bg)
        path = os.path.join(out_dir, f"bg{bg}_z{Z}.npz")
        np.savez_compressed(path, entries=entries, info=info, codewords=cw, Z=Z, bg=bg)
        print(path, len(entries), "circulants", os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
