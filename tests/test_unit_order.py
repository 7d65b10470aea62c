"""The matching's processing order (csrc/unit_order.h, run by the host and
the device router) is the same permutation as the C++ library's std::sort
on the same comparator, ties included (compiled with g++, no GPU)."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_unit_order_equals_std_sort(tmp_path):
    exe = tmp_path / "unit_order_check"
    subprocess.run(["g++", "-O2", "-std=c++17", os.path.join(HERE, "unit_order_check.cpp"),
                    "-o", str(exe)], check=True, capture_output=True, timeout=300)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True, timeout=300)
    assert out.stdout.startswith("ok")
