"""The C++ interface compiles as C++11 with warnings as errors and links
against the library without the CUDA toolkit (no device needed); the
generic Sampler<T> header with device moves compiles with nvcc for sm_100a
(no device needed either)."""
import os
import subprocess

import pytest

from facade_util import LIBDIR, compile_facade


def test_facade_compiles(tmp_path):
    compile_facade(str(tmp_path), link=False)


def test_facade_links(tmp_path):
    if not os.path.exists(os.path.join(LIBDIR, "libvsmc_cuda.so")):
        pytest.skip("libvsmc_cuda.so not built")
    exe = compile_facade(str(tmp_path))
    # no arguments: usage status, no device call
    r = subprocess.run([exe], capture_output=True)
    assert r.returncode == 2


def test_generic_sampler_compiles(tmp_path):
    from test_gpu_generic import compile_generic

    if not os.path.exists(os.path.join(LIBDIR, "libvsmc_cuda.so")):
        pytest.skip("libvsmc_cuda.so not built")
    exe = compile_generic(str(tmp_path))
    assert os.path.exists(exe)
