"""The slice plan of the host-buffer calls, checked on the host: the plan's
header is plain C++, compiled here with g++ together with
tests/host_plan/check_plan.cpp, which walks every batch size below 20,000 and
a set of large ones with 0..8 wanted slices."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ is not installed")
def test_every_slice_is_in_range_and_non_empty(tmp_path):
    exe = str(tmp_path / "check_plan")
    subprocess.run(["g++", "-std=c++17", "-O2", "-o", exe, os.path.join(HERE, "host_plan", "check_plan.cpp")],
                   check=True, capture_output=True, text=True)
    res = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert res.returncode == 0, res.stdout + res.stderr
    assert res.stdout.strip().endswith("bad 0"), res.stdout
