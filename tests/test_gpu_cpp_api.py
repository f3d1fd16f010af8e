"""Build and run tests/cpp/test_stage_api.cpp: the C++ drop-in classes of
include/skyweaver_b200.hpp exercised like the reference's gtest fixtures and
checked against the oracle library."""
import os
import shutil
import subprocess

import pytest

from conftest import GOLDEN, REPO

pytestmark = pytest.mark.gpu


def _build(oracle):
    out_dir = os.path.join(REPO, "skyweaver_b200", "_build")
    os.makedirs(out_dir, exist_ok=True)
    exe = os.path.join(out_dir, "test_stage_api")
    cuda = os.path.dirname(os.path.dirname(shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"))
    lib_dir = os.path.join(REPO, "skyweaver_b200")
    cmd = ["g++", "-std=c++17", "-O2", os.path.join(REPO, "tests", "cpp", "test_stage_api.cpp"),
           f"-I{REPO}/include", f"-I{cuda}/include", f"-L{lib_dir}", "-lskyweaver_b200",
           f"-L{REPO}/oracle", "-lswb_oracle", f"-L{cuda}/lib64", "-lcudart",
           f"-Wl,-rpath,{lib_dir}", f"-Wl,-rpath,{REPO}/oracle", "-o", exe]
    subprocess.check_call(cmd)
    return exe


def test_cpp_stage_api(cuda, oracle):
    exe = _build(oracle)
    scratch = os.path.join(REPO, "skyweaver_b200", "_build", "cpp_scratch")
    shutil.rmtree(scratch, ignore_errors=True)
    os.makedirs(scratch)
    r = subprocess.run([exe, GOLDEN, scratch], capture_output=True, text=True, timeout=300)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "ALL PASS" in r.stdout
