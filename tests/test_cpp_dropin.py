"""The C++ drop-in (include/fem/*.hpp over libfem_b200): the reference's own
test cases, restated in tests/cpp/, compiled with g++ against the drop-in
headers and the library -- the way a user of the reference switches over."""
import glob
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CPP = os.path.join(ROOT, "tests", "cpp")
BIN = os.path.join(CPP, "_build", "fem_cpp_tests")


def _build():
    from fe_demo_cpp_b200 import build as b
    lib = b.build()
    srcs = sorted(glob.glob(os.path.join(CPP, "*.cpp")))
    deps = srcs + glob.glob(os.path.join(CPP, "*.hpp")) + glob.glob(os.path.join(ROOT, "include", "**", "*.h*"),
                                                                     recursive=True) + [lib]
    if os.path.exists(BIN) and all(os.path.getmtime(d) <= os.path.getmtime(BIN) for d in deps):
        return BIN
    os.makedirs(os.path.dirname(BIN), exist_ok=True)
    libdir = os.path.dirname(lib)
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-I", os.path.join(ROOT, "include", "fem"), *srcs,
           "-L", libdir, "-lfem_b200", f"-Wl,-rpath,{libdir}", "-o", BIN]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stdout + res.stderr
    return BIN


def _run(mode):
    exe = _build()
    res = subprocess.run([exe, mode], capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stdout + res.stderr
    return res.stdout


def test_cpp_dropin_builds_and_host_cases_pass(fem):
    out = _run("--cpu")
    assert "0 failed" in out, out


@pytest.mark.gpu
def test_cpp_dropin_gpu_cases_pass(fem, cuda):
    out = _run("--gpu")
    assert "0 failed" in out, out
