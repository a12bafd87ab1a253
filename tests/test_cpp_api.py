"""The C++ helpers of include/mgpusort.hpp and the C ABI, called from C++ the
way the reference's example programs call them (tests/cpp/cpp_api_test.cpp),
built here against libmgpusort_b200.so."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "cpp_api_test.cpp")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def build_binary(out_dir, lib):
    exe = os.path.join(out_dir, "cpp_api_test")
    libdir = os.path.join(ROOT, "mgpu_old_b200")
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Wno-pedantic",
                    "-I", os.path.join(ROOT, "include"), "-I", os.path.join(CUDA, "include"),
                    SRC, "-L", libdir, "-lmgpusort_b200",
                    "-L", os.path.join(CUDA, "lib64", "stubs"), "-lcuda",
                    f"-Wl,-rpath,{libdir}", "-o", exe], check=True)
    return exe


def test_cpp_api_compiles(lib, tmp_path):
    assert os.path.exists(build_binary(str(tmp_path), lib))


@pytest.mark.gpu
def test_cpp_api_runs(lib, tmp_path):
    exe = build_binary(str(tmp_path), lib)
    env = dict(os.environ)
    env.pop("CUDA_VISIBLE_DEVICES", None) if env.get("CUDA_VISIBLE_DEVICES") == "" else None
    out = subprocess.run([exe], capture_output=True, text=True, timeout=300, env=env)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "cpp_api_test: OK" in out.stdout
