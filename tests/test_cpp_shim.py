"""The header-only C++ driver layer (include/ctstereo.hpp) compiled with g++
against libctstereo.so and driven like the reference's CDriver classes
(Configure -> ProcessKernel -> CopyInto): argument checks on the CPU, and on
the GPU every driver on a pair with a known integer shift."""
import os
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG = ROOT / "module.clutec.cuda_b200"
CUDA = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))


@pytest.fixture(scope="module")
def shim_test(ct, tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("no g++")
    exe = tmp_path_factory.mktemp("shim") / "shim_test"
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror",
           "-I", str(ROOT / "include"), "-I", str(CUDA / "include"),
           str(ROOT / "tests" / "cpp" / "shim_test.cpp"),
           "-L", str(PKG), "-lctstereo", "-L", str(CUDA / "lib64"), "-lcudart",
           f"-Wl,-rpath,{PKG}", f"-Wl,-rpath,{CUDA / 'lib64'}", "-o", str(exe)]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def _run(exe, *args, timeout=120):
    r = subprocess.run([str(exe), *args], capture_output=True, text=True, timeout=timeout)
    print(r.stdout)
    return r


def test_shim_rejects_unbuilt_reference_options(shim_test):
    r = _run(shim_test, "cpu")
    assert r.returncode == 0, r.stdout + r.stderr


@pytest.mark.gpu
def test_shim_drivers_on_a_known_shift(shim_test, cuda):
    r = _run(shim_test, "gpu", str(PKG / "confnet_census128.f32"))
    assert r.returncode == 0, r.stdout + r.stderr
