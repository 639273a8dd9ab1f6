"""The reference's test program, re-expressed against the C++ drop-in header
(tests/cpp/sort512cuda_test.cpp), compiled here and run on the GPU."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.gpu
def test_reference_test_program_on_dropin(s512, tmp_path):
    exe = str(tmp_path / "sort512cuda_test")
    libdir = os.path.dirname(s512.LIB_PATH)
    r = subprocess.run(["/usr/bin/g++", "-O2", "-std=c++14", "-I" + os.path.join(ROOT, "include"),
                        os.path.join(ROOT, "tests", "cpp", "sort512cuda_test.cpp"), "-L" + libdir, "-lsort512cuda",
                        "-Wl,-rpath," + libdir, "-o", exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([exe], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-2000:]
    assert "All tests passed" in r.stdout
