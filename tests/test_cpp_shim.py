"""The C++ mirror of the operator classes (include/megastation_b200.hpp):
it compiles against the C ABI on the CPU, and on a GPU it reproduces the
reference's golden unit-test cases through the same call shapes."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA = "/usr/local/cuda"


def _compile(out):
    cxx = shutil.which("g++") or "/usr/bin/g++"
    cmd = [cxx, "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), "-I", f"{CUDA}/include",
           os.path.join(ROOT, "tests", "cpp", "shim_golden.cpp"), "-o", out,
           "-L", os.path.join(ROOT, "megastation_b200"), "-lmegastation_b200",
           f"-Wl,-rpath,{os.path.join(ROOT, 'megastation_b200')}",
           "-L", f"{CUDA}/lib64", "-lcudart", f"-Wl,-rpath,{CUDA}/lib64"]
    subprocess.check_call(cmd)


def test_shim_compiles_and_links(tmp_path):
    _compile(str(tmp_path / "shim_golden"))


@pytest.mark.gpu
def test_shim_reproduces_golden_cases(tmp_path):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    exe = str(tmp_path / "shim_golden")
    _compile(exe)
    r = subprocess.run([exe, os.path.join(ROOT, "tests", "golden")], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "all golden cases match" in r.stdout
