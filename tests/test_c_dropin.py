"""The drop-in swap a C user of hmat_lib makes: tests/c_dropin_caller.c is
compiled with gcc against include/hmat_lib/*.h and linked to
libhodlr_b200.so (no Python in between).  On CPU: it compiles and links, so
the headers are valid C and the library exports every symbol the program
uses.  On the GPU: it runs -- builds a tree with dense_to_tree_hodlr,
multiplies it by a vector, by dense blocks (H X, H^T X, X H with padded
leading dimensions, library-allocated results) and by itself
(multiply_hodlr_hodlr), checks each against a dense product it computes
itself, and frees everything (the calling pattern of hmat_lib dev/test.c)."""
import os
import subprocess

import pytest

from hmat_lib_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "c_dropin_caller.c")


def _compile(tmp_path):
    exe = os.path.join(str(tmp_path), "c_dropin_caller")
    libdir = os.path.dirname(abi.lib_path())
    cmd = ["gcc", "-std=c11", "-O1", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), SRC,
           "-L", libdir, "-lhodlr_b200", f"-Wl,-rpath,{libdir}", "-lm", "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    return exe


def test_c_caller_compiles_and_links(tmp_path):
    assert os.path.exists(_compile(tmp_path))


@pytest.mark.gpu
def test_c_caller_runs_on_gpu(tmp_path):
    exe = _compile(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "ALL OK" in r.stdout
