"""The C++ adapter (include/ilc_backend.hpp) compiles against the C ABI and,
on a GPU, drives the nn8 backend and a projection like illcrawl's callers."""
import os
import subprocess

import pytest

from conftest import ROOT

SRC = os.path.join(ROOT, "tests", "cpp", "adapter_demo.cpp")
EXE = os.path.join(ROOT, "_build", "adapter_demo")


def _compile(cuda_lib):
    os.makedirs(os.path.dirname(EXE), exist_ok=True)
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    subprocess.run([cxx, "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), SRC, "-o",
                    EXE, "-L", os.path.dirname(cuda_lib), "-lilcuda",
                    f"-Wl,-rpath,{os.path.dirname(cuda_lib)}"], check=True)


def test_adapter_compiles_and_fails_loudly_without_gpu(cuda_lib):
    import torch
    _compile(cuda_lib)
    if torch.cuda.is_available():
        pytest.skip("GPU present: covered by the gpu test")
    r = subprocess.run([EXE], capture_output=True, text=True)
    assert r.returncode == 2 and "no usable CUDA device" in r.stdout


@pytest.mark.gpu
def test_adapter_runs_on_gpu(cuda_lib):
    _compile(cuda_lib)
    r = subprocess.run([EXE], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.startswith("ok ")
