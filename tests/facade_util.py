"""Compiles tests/cpp/facade_main.cpp against the C++ interface
(include/vsmc_b200/vsmc_cuda.hpp) and libvsmc_cuda.so with the host C++
compiler only: the interface needs no CUDA toolkit."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "facade_main.cpp")
LIBDIR = os.path.join(ROOT, "vsmc_b200", "lib")


def compile_facade(out_dir, link=True):
    exe = os.path.join(out_dir, "facade_main" if link else "facade_main.o")
    cmd = [os.environ.get("CXX", "g++"), "-std=c++11", "-O2", "-Wall", "-Wextra", "-Werror",
           "-I", os.path.join(ROOT, "include"), SRC, "-o", exe]
    if link:
        cmd += ["-L", LIBDIR, "-lvsmc_cuda", f"-Wl,-rpath,{LIBDIR}"]
    else:
        cmd.insert(1, "-c")
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe
