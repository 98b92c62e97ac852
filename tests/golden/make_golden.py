"""Copies the MegaStation unit-test golden vectors for the hot path into
tests/golden/ so that the parity tests run where the reference tree is not
mounted.  The files are the reference's own fixtures, byte for byte:

  test/fft/{zachu,zachu_shift,short_in,complex_out,fft_in,fft_out,ifft_in,ifft_out}.data
      (read by test/fft/test_fft.cc:10-215)
  test/beamform/{csi_in,csi_out,precoder}.data   (test/beamform/test_beamform.cc:19-95)
  test/sgemv/{csi,bsVec,equalize,prec,ueVec,precoded}.data (test/sgemv/test_sgemv.cc:32-196)

Usage: python tests/golden/make_golden.py /path/to/MegaStation
(or with the tree's location in the MEGASTATION_REF environment variable)
"""
import os
import shutil
import sys

FILES = {
    "fft": ["zachu", "zachu_shift", "short_in", "complex_out", "fft_in", "fft_out", "ifft_in", "ifft_out"],
    "beamform": ["csi_in", "csi_out", "precoder"],
    "sgemv": ["csi", "bsVec", "equalize", "prec", "ueVec", "precoded"],
}


def main(ref_root):
    here = os.path.dirname(os.path.abspath(__file__))
    for sub, names in FILES.items():
        os.makedirs(os.path.join(here, sub), exist_ok=True)
        for n in names:
            src = os.path.join(ref_root, "test", sub, n + ".data")
            dst = os.path.join(here, sub, n + ".data")
            shutil.copyfile(src, dst)
            print(dst, os.path.getsize(dst))


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("MEGASTATION_REF")
    if not root:
        sys.exit("usage: make_golden.py <MegaStation tree> (or set MEGASTATION_REF)")
    main(root)
