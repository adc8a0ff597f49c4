"""A C program compiled against the unchanged include/libfive.h and linked
to lib/libfive.so (tests/capi/api_replay.c: the C-API cases of
libfive/test/api.cpp).  The build and link run on the CPU; running it needs
the GPU."""
import os
import subprocess

import pytest

from libfive_b200 import build

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def compile_replay(tmp_path):
    exe = str(tmp_path / "api_replay")
    libdir = os.path.dirname(build.LIB)
    cmd = ["gcc", "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
           os.path.join(HERE, "capi", "api_replay.c"), "-o", exe, "-L", libdir, "-lfive",
           "-Wl,-rpath," + libdir, "-lm"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_c_program_builds_and_links(tmp_path):
    exe = compile_replay(tmp_path)
    # every symbol the program uses resolves against lib/libfive.so
    r = subprocess.run(["ldd", "-r", exe], capture_output=True, text=True)
    assert "undefined symbol" not in r.stdout + r.stderr


@pytest.mark.gpu
def test_c_program_runs(gpu, tmp_path):
    exe = compile_replay(tmp_path)
    r = subprocess.run([exe, str(tmp_path / "sphere.stl")], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "api_replay ok" in r.stdout
