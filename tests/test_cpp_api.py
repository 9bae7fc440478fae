"""The C++ drop-in headers (include/stereo/*.h) compile against the C ABI and
map statuses to the reference's exception types."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "api_surface.cpp")
LIBDIR = os.path.join(ROOT, "lumenstereo_b200")


def build_binary(tmp_path):
    cxx = shutil.which("g++")
    if not cxx:
        pytest.skip("no C++ compiler")
    exe = str(tmp_path / "api_surface")
    subprocess.run([cxx, "-std=c++17", "-O1", "-Wall", "-I", os.path.join(ROOT, "include"), SRC,
                    "-L", LIBDIR, "-llumen_sgbm", f"-Wl,-rpath,{LIBDIR}", "-o", exe], check=True)
    return exe


def test_cpp_headers_cpu(tmp_path):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("CPU variant: runs where no GPU is visible")
    except ImportError:
        pass
    exe = build_binary(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 0 and "ok" in r.stdout, r.stdout + r.stderr


@pytest.mark.gpu
def test_cpp_headers_gpu(tmp_path):
    exe = build_binary(tmp_path)
    r = subprocess.run([exe, "gpu"], capture_output=True, text=True)
    assert r.returncode == 0 and "ok" in r.stdout, r.stdout + r.stderr
