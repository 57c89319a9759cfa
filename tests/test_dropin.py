"""The drop-in header: a user kernel that calls mm->malloc / mm->free itself."""
import os
import subprocess

import pytest

from ouroboros_b200 import build

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
EXE = os.path.join(ROOT, "ouroboros_b200", "_lib", "dropin_user_kernel")


def _compile():
    lib = build.build()
    if os.path.exists(EXE) and os.path.getmtime(EXE) >= max(
            os.path.getmtime(lib), os.path.getmtime(os.path.join(HERE, "dropin", "user_kernel.cu")),
            os.path.getmtime(os.path.join(ROOT, "include", "ouroboros_b200.cuh"))):
        return EXE
    cmd = [build.nvcc(), "-std=c++17", "-O3", "-gencode", "arch=compute_100a,code=sm_100a",
           "-I", os.path.join(ROOT, "include"), os.path.join(HERE, "dropin", "user_kernel.cu"),
           "-L", os.path.dirname(lib), "-louroboros_b200", f"-Xlinker=-rpath,{os.path.dirname(lib)}", "-o", EXE]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr[-3000:]
    return EXE


def test_dropin_compiles():
    assert os.path.exists(_compile())


@pytest.mark.gpu
def test_dropin_user_kernel_churn():
    exe = _compile()
    res = subprocess.run([exe, "592", "8"], capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stdout + res.stderr
    assert res.stdout.count('"bad": 0') == 6
