"""The C++ drop-in header (include/srk_b200.hpp) used from a C++ caller the way
the reference's op_test() slot is: compiled here, run on the GPU."""
import os
import subprocess

import pytest

from shrinkage_full_tests_b200 import build as B

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "dropin_training.cu")


def compile_driver(tmp_path):
    exe = str(tmp_path / "dropin_training")
    lib = B.build()
    cmd = [B.NVCC, "-std=c++17", "-O2", "-gencode", "arch=compute_100a,code=sm_100a", "-I" + os.path.join(ROOT, "include"),
           SRC, "-o", exe, "-L" + os.path.dirname(lib), "-lsrk_b200", "-Xlinker", "-rpath=" + os.path.dirname(lib)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_cpp_driver_compiles(tmp_path):
    assert os.path.exists(compile_driver(tmp_path))


@pytest.mark.gpu
def test_cpp_dropin_training_forward(tmp_path, torch_cuda):
    exe = compile_driver(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "PASS" in r.stdout
