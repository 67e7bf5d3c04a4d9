"""The request server's admission rule on the CPU.

tests/admission_check.cpp drives uncertaintyte_b200/csrc/admission.h (the
rule server.cu uses) through seeded simulations of workers that hold two
workspaces each, and checks that the bytes held stay within the budget, that
each worker's commitment matches what it holds, and that every request is
admitted once and finishes. It is built with AddressSanitizer and
UndefinedBehaviorSanitizer, so a reference into the request queue kept past an
erase fails the test too.
"""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "uncertaintyte_b200", "csrc")


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_admission_rule(tmp_path):
    exe = str(tmp_path / "admission_check")
    subprocess.run(["g++", "-std=c++17", "-O1", "-g", "-fsanitize=address,undefined",
                    "-fno-sanitize-recover=undefined", "-I", CSRC, os.path.join(HERE, "admission_check.cpp"),
                    "-o", exe], check=True)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "admission ok" in out.stdout
