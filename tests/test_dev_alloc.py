"""Host test of the allocation layer (pi-compute_b200/csrc/dev_alloc.h): deferred frees inside the
pi calls, their flush, their cap, the retry after an allocation fails for want of memory, and the
injected allocation failure, against a fake CUDA runtime compiled into the test program
(tests/native/dev_alloc_test.cpp). No GPU."""
import os
import shutil
import subprocess

import pytest

from helpers import ROOT

CUDA_INC = "/usr/local/cuda/include"


@pytest.mark.skipif(not (shutil.which("g++") and os.path.isdir(CUDA_INC)), reason="needs g++ and the CUDA headers")
def test_deferred_frees_against_a_fake_runtime(tmp_path):
    exe = str(tmp_path / "dev_alloc_test")
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", CUDA_INC, "-I", os.path.join(ROOT, "pi-compute_b200", "csrc"),
                    os.path.join(ROOT, "tests", "native", "dev_alloc_test.cpp"), "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stderr
