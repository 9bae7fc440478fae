"""The C++ drop-in headers (include/stereo/*.h) compile against the C ABI and
map statuses to the reference's exception types."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "api_surface.cpp")
LIBDIR = os.path.join(ROOT, "lumenstereo_b200")


SRC_CV = os.path.join(ROOT, "tests", "cpp", "api_cvmat.cpp")
FAKE_CV = os.path.join(ROOT, "tests", "cpp", "fake_opencv")


def build_binary(tmp_path, src=SRC, extra_includes=()):
    cxx = shutil.which("g++")
    if not cxx:
        pytest.skip("no C++ compiler")
    exe = str(tmp_path / os.path.splitext(os.path.basename(src))[0])
    inc = []
    for d in extra_includes:
        inc += ["-I", d]
    subprocess.run([cxx, "-std=c++17", "-O1", "-Wall", *inc, "-I", os.path.join(ROOT, "include"),
                    src, "-L", LIBDIR, "-llumen_sgbm", f"-Wl,-rpath,{LIBDIR}", "-o", exe],
                   check=True)
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


def _no_gpu_visible():
    try:
        import torch
        return not torch.cuda.is_available()
    except ImportError:
        return True


def test_cpp_cvmat_forms_cpu(tmp_path):
    """The reference's cv::Mat / CameraParams signatures compile (against a
    stand-in cv::Mat) and reject bad maps before touching the device."""
    if not _no_gpu_visible():
        pytest.skip("CPU variant: runs where no GPU is visible")
    exe = build_binary(tmp_path, SRC_CV, (FAKE_CV,))
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 0 and "ok" in r.stdout, r.stdout + r.stderr


@pytest.mark.gpu
def test_cpp_cvmat_forms_gpu(tmp_path):
    """Every cv::Mat form equals the raw-pointer form of the same call."""
    exe = build_binary(tmp_path, SRC_CV, (FAKE_CV,))
    r = subprocess.run([exe, "gpu"], capture_output=True, text=True)
    assert r.returncode == 0 and "ok" in r.stdout, r.stdout + r.stderr
