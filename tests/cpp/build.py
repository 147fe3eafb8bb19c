"""Builds tests/cpp/fcib_solver_main with g++ against include/ and forte_b200/libfcib200.so (rpath
set, so the binary finds the in-tree library).  Returns the binary's path."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def build(out_dir=None):
    out_dir = out_dir or HERE
    exe = os.path.join(out_dir, "fcib_solver_main")
    libdir = os.path.join(ROOT, "forte_b200")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-I", os.path.join(ROOT, "include"),
           os.path.join(HERE, "fcib_solver_main.cpp"), "-L", libdir, "-lfcib200", f"-Wl,-rpath,{libdir}",
           "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("g++ failed:\n" + r.stdout + r.stderr)
    return exe
