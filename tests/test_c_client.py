"""The drop-in boundary from C: tests/c_client/dropin_client.c is written
against the reference's public API (include/gooseberry.h: names, argument
order, GOOSEBERRY_SUCCESS = 1) and links with libgooseberry_b200.so.  It
compiles as C99 and as C++ with warnings as errors; on a GPU it runs SpMV,
multi-column SpMV, CG, Cuthill-McKee and a sparse permutation and checks
their results."""
from __future__ import annotations

import os
import shutil
import subprocess

import pytest

import gooseberry_b200 as gb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "c_client", "dropin_client.c")
INC = os.path.join(ROOT, "include")
LIBDIR = os.path.dirname(gb.LIB_PATH)


def _cc():
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    return cc


def _build(tmp_path):
    gb.lib()  # the library exists (raises otherwise)
    exe = str(tmp_path / "dropin_client")
    subprocess.run([_cc(), "-std=c99", "-Wall", "-Wextra", "-Werror", "-I", INC, SRC,
                    "-L", LIBDIR, "-lgooseberry_b200", f"-Wl,-rpath,{LIBDIR}", "-lm", "-o", exe],
                   check=True, capture_output=True, text=True)
    return exe


def test_client_compiles_as_c_and_cpp_and_links(tmp_path):
    _build(tmp_path)
    cxx = shutil.which("g++")
    if cxx:
        subprocess.run([cxx, "-x", "c++", "-std=c++17", "-Wall", "-Werror", "-I", INC,
                        "-fsyntax-only", SRC], check=True, capture_output=True, text=True)


@pytest.mark.gpu
def test_client_runs(tmp_path):
    exe = _build(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert "dropin ok" in r.stdout
