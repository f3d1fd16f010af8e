"""Build and run tests/cpp/test_host_api.cpp on the CPU: the host-side C++
classes of include/skyweaver_b200.hpp (dedispersion plan, PipelineConfig,
DescribedVector views, the coherent dedisperser's configuration checks),
which make no CUDA call."""
import os
import shutil
import subprocess

from conftest import REPO


def test_cpp_host_api(tmp_path):
    from skyweaver_b200 import _lib
    if not os.path.exists(_lib.LIB_PATH):
        from skyweaver_b200 import build
        build.build()
    cuda = os.path.dirname(os.path.dirname(shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"))
    lib_dir = os.path.dirname(_lib.LIB_PATH)
    exe = str(tmp_path / "test_host_api")
    subprocess.check_call(
        ["g++", "-std=c++17", "-O1", os.path.join(REPO, "tests", "cpp", "test_host_api.cpp"),
         f"-I{REPO}/include", f"-I{cuda}/include", f"-L{lib_dir}", "-lskyweaver_b200",
         f"-L{cuda}/lib64", "-lcudart", f"-Wl,-rpath,{lib_dir}", f"-Wl,-rpath,{cuda}/lib64",
         "-o", exe])
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "ALL PASS" in r.stdout, r.stdout
