"""Compiled callers of libsbb.so (tests/c): a C program through
include/sbb_spmv.h and a C++ program that declares the entry points with the
reference header's C++ linkage, built here with gcc / g++ and run as the
reference's own test driver would run (SparseBLAS/test/dspmv_test.cu).
Without a GPU only their host-only mode runs (argument checks, helpers)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "sparse-blas_b200", "sbb")
PROGRAMS = [("dropin_test.c", False), ("dropin_cxx_test.cpp", True)]


def _build(tmp_path, src, cxx):
    cc = shutil.which("g++" if cxx else "gcc")
    if cc is None:
        pytest.skip("no host compiler")
    if not os.path.exists(os.path.join(LIBDIR, "libsbb.so")):
        pytest.fail("libsbb.so is not built (make -C sparse-blas_b200)")
    exe = tmp_path / (src.split(".")[0] + ".bin")
    cmd = [cc, "-O2", "-std=c++17" if cxx else "-std=c99", "-Wall", f"-I{ROOT}/include",
           os.path.join(ROOT, "tests", "c", src), f"-L{LIBDIR}", "-lsbb",
           f"-Wl,-rpath,{LIBDIR}", "-lm", "-o", str(exe)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


@pytest.mark.parametrize("src,cxx", PROGRAMS, ids=[p[0] for p in PROGRAMS])
def test_compiled_callers_host_only(tmp_path, src, cxx):
    exe = _build(tmp_path, src, cxx)
    r = subprocess.run([str(exe), "--host-only"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "host-only ok" in r.stdout


@pytest.mark.gpu
@pytest.mark.parametrize("src,cxx", PROGRAMS, ids=[p[0] for p in PROGRAMS])
def test_compiled_callers_on_gpu(cuda, tmp_path, src, cxx):
    exe = _build(tmp_path, src, cxx)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "ok" in r.stdout
