"""A C program (tests/c_caller/lifecycle.c) built against include/xamg_c_api.h
with the system C compiler and linked to lib/libxamg_c_api.so as INTEGRATION.md
describes: the header compiles as C99 with warnings as errors, the program
links, and on a GPU it runs the whole XAMG C lifecycle to its tolerances."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "softx-d-21-00014_b200", "lib")
SRC = os.path.join(ROOT, "tests", "c_caller", "lifecycle.c")


def build(tmp_path):
    exe = str(tmp_path / "lifecycle")
    subprocess.check_call(["cc", "-std=c99", "-Wall", "-Wextra", "-Werror",
                           "-Wno-unused-parameter", "-I", os.path.join(ROOT, "include"), SRC,
                           "-o", exe, "-L", LIBDIR, "-lxamg_c_api", "-lm",
                           f"-Wl,-rpath,{LIBDIR}"])
    return exe


def test_c_program_compiles_and_links(xamg, tmp_path):
    exe = build(tmp_path)
    out = subprocess.check_output(["ldd", exe], text=True)
    assert os.path.join(LIBDIR, "libxamg_c_api.so") in out


@pytest.mark.gpu
def test_c_program_runs_the_lifecycle(xamg, tmp_path):
    exe = build(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "lifecycle:" in r.stdout
