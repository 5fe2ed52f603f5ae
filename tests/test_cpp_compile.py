"""The C++ class surface (include/sph_swe/sph_swe.hpp) and the programs built
on it compile and link against libsphgpu.so without a GPU (the GPU tests run
them)."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "sph_swe_b200")


@pytest.fixture(scope="module")
def built():
    from sph_swe_b200 import build

    build.build()
    return True


@pytest.mark.parametrize("prog", ["classes_check.cpp", "classes_check_cplx.cpp", "rexi_pole_check.cpp"])
def test_cpp_program_compiles(built, tmp_path, prog):
    out = str(tmp_path / prog.replace(".cpp", ""))
    r = subprocess.run(["/usr/bin/g++", "-std=c++17", "-O1", "-Wall", "-I", os.path.join(ROOT, "include"), "-I",
                        "/usr/local/cuda/include", os.path.join(ROOT, "tests", "cpp", prog), "-o", out, "-L", PKG,
                        "-lsphgpu", "-L", "/usr/local/cuda/lib64", "-lcudart"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert "warning" not in r.stderr, r.stderr


def test_sh_example_is_built(built):
    assert os.access(os.path.join(PKG, "sh_example"), os.X_OK)
