"""CPU checks of code the CUDA kernels share with the host.

The border-initialisation gather (csrc/border.cuh) is __host__ __device__; it
is compiled here with g++ and compared with the oracle's restatement of the
reference's write order on randomised masks, so the word-boundary and
row/slice-pair ordering rules are covered without a GPU.
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def hostlib(tmp_path_factory):
    out = tmp_path_factory.mktemp("hostlogic") / "libborder_host.so"
    src = os.path.join(ROOT, "tests", "border_host.cpp")
    inc = os.path.join(ROOT, "distance-occlusion_b200", "csrc")
    subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-I" + inc, src, "-o", str(out)], check=True)
    return C.CDLL(str(out))


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def _mask(O, rng, dims, p, garbage):
    m = O.bool_to_mask(rng.random(tuple(reversed(dims))) < p)
    w = dims[0]
    if garbage and w % 32:
        rows = m.reshape(-1, (w + 31) // 32)
        rows[:, -1] |= np.uint32(0xFFFFFFFF) << np.uint32(w % 32)
        m = rows.reshape(-1)
    return m


@pytest.mark.parametrize("dims", [(1, 1), (1, 4), (5, 1), (31, 5), (32, 6), (33, 7), (64, 10), (65, 3), (130, 40)])
def test_border2_gather_matches_oracle(O, hostlib, dims):
    rng = np.random.default_rng(sum(dims))
    w, h = dims
    for p in (0.0, 0.02, 0.2, 0.5, 0.8, 1.0):
        for garbage in (False, True):
            m = _mask(O, rng, dims, p, garbage)
            got = np.empty((h, w, 2), dtype=np.int16)
            hostlib.host_border_2d(C.c_int(w), C.c_int(h), _p(m), _p(got))
            np.testing.assert_array_equal(got, O.border_init(m, dims), err_msg=f"p={p}")


@pytest.mark.parametrize("dims", [(1, 1, 1), (1, 3, 4), (4, 1, 3), (3, 4, 1), (31, 5, 4), (32, 4, 5), (33, 6, 3),
                                  (65, 4, 6), (70, 9, 8), (40, 1, 7), (40, 7, 1)])
def test_border3_gather_matches_oracle(O, hostlib, dims):
    rng = np.random.default_rng(sum(dims) + 7)
    w, h, d = dims
    for p in (0.0, 0.02, 0.2, 0.5, 0.8, 1.0):
        for garbage in (False, True):
            m = _mask(O, rng, dims, p, garbage)
            got = np.empty((d, h, w, 3), dtype=np.int16)
            hostlib.host_border_3d(C.c_int(w), C.c_int(h), C.c_int(d), _p(m), _p(got))
            np.testing.assert_array_equal(got, O.border_init(m, dims), err_msg=f"p={p}")
