"""The header-only C++ projector classes (include/reconnet_b200_projector.hpp,
the reference's Projector / DistanceDrivenFan / DistanceDrivenTomo interface,
ReconNet4D/Projector.h:8-63, DistanceDriven.h:3-30): the header compiles on
the CPU, and on the GPU a C++ program built against the library checks the
classes against the plain C ABI (tests/cpp/projector_class.cpp)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "projector_class.cpp")
CUDA_INC = "/usr/local/cuda/include"
CUDA_LIB = "/usr/local/cuda/lib64"


def _gxx():
    gxx = shutil.which("g++")
    if gxx is None or not os.path.isdir(CUDA_INC):
        pytest.skip("g++ or the CUDA headers are not available")
    return gxx


def test_projector_header_compiles():
    r = subprocess.run([_gxx(), "-std=c++17", "-Wall", "-Werror", "-fsyntax-only", "-I" + os.path.join(ROOT, "include"),
                        "-I" + CUDA_INC, SRC], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


@pytest.mark.gpu
def test_projector_classes_match_c_abi(tmp_path):
    from reconnet_b200 import _native  # noqa: F401  (the library is built and loadable)
    libdir = os.path.join(ROOT, "reconnet_b200", "_lib")
    exe = str(tmp_path / "projector_class")
    r = subprocess.run([_gxx(), "-std=c++17", "-O2", "-I" + os.path.join(ROOT, "include"), "-I" + CUDA_INC, SRC,
                        "-L" + libdir, "-lreconnet_b200", "-L" + CUDA_LIB, "-lcudart", "-Wl,-rpath," + libdir,
                        "-o", exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    run = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert run.returncode == 0 and run.stdout.strip().endswith("OK"), run.stdout + run.stderr
