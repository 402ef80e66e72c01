"""CPU checks of the EDT's lower-envelope path (csrc/hull.cuh).

The line kernel sends tiles whose cells lie far from the other state (sparse
or empty volumes) to the lower-envelope routines.  They are __host__
__device__; compiled here with g++, they run on split tiles built the way the
kernel builds them (F_s holds a state-s cell's own value, 0 for the other
state, the sentinel for "none" and past the line end) and must give, for
every cell of state s, exactly min over p' of G_s(p') + (p - p')^2 -- the
brute-force 1D transform -- including the cells with no candidate at all.
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def hull(tmp_path_factory):
    out = tmp_path_factory.mktemp("hull") / "libhull_host.so"
    src = os.path.join(ROOT, "tests", "edt_hull_host.cpp")
    inc = os.path.join(ROOT, "distance-occlusion_b200", "csrc")
    subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-I" + inc, src, "-o", str(out)], check=True)
    return C.CDLL(str(out))


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def make_tile(states, vals, dtype):
    """states, vals: (n, TX); vals 0 = none.  Returns F0, F1 of 32*ceil(n/32) rows."""
    n, tx = states.shape
    rows = 32 * ((n + 31) // 32)
    sent = 0x7FFF if dtype == np.uint16 else 0x7FFFFFFF
    own = np.where(vals == 0, sent, vals).astype(np.int64)
    F0 = np.full((rows, tx), sent, np.int64)
    F1 = np.full((rows, tx), sent, np.int64)
    F0[:n] = np.where(states == 0, own, 0)
    F1[:n] = np.where(states == 1, own, 0)
    return F0.astype(dtype), F1.astype(dtype)


def brute(states, vals, dtype):
    n, tx = states.shape
    sq = (lambda v: v * v) if dtype == np.uint16 else (lambda v: v)
    best = np.zeros((n, tx), np.int64)
    none = np.zeros((n, tx), bool)
    pos = np.arange(n)
    for c in range(tx):
        for p in range(n):
            s = states[p, c]
            g = np.where(states[:, c] != s, 0, np.where(vals[:, c] == 0, -1, sq(vals[:, c].astype(np.int64))))
            ok = g >= 0
            if not ok.any():
                none[p, c] = True
                continue
            best[p, c] = (g[ok] + (pos[ok] - p) ** 2).min()
    return best, none


def run_case(hull, states, vals, dtype, sb=32):
    F0, F1 = make_tile(states, vals, dtype)
    n, tx = states.shape
    rows = F0.shape[0]
    best = np.zeros((rows, tx), np.uint32)
    none = np.zeros((rows, tx), np.uint8)
    fn = hull.hull_tile_u16 if dtype == np.uint16 else hull.hull_tile_u32
    fn(C.c_int(n), C.c_int(tx), _p(np.ascontiguousarray(F0)), _p(np.ascontiguousarray(F1)), _p(best), _p(none),
       C.c_int(sb))
    want, want_none = brute(states, vals, dtype)
    np.testing.assert_array_equal(none[:n].astype(bool), want_none)
    np.testing.assert_array_equal(np.where(want_none, 0, best[:n]), np.where(want_none, 0, want))


CASES = ["random", "sparse", "empty", "full", "constant", "runs", "single", "large"]


def gen(kind, n, tx, dtype, rng):
    hi = 300 if dtype == np.uint16 else 90000
    if kind == "large":        # own values near the largest a 16384-cell side gives
        top = 16383 if dtype == np.uint16 else 2 * 16383 * 16383
        st = (rng.random((n, tx)) < 0.3).astype(np.int64)
        v = top - rng.integers(0, top // 50, (n, tx))
    elif kind == "random":
        st = (rng.random((n, tx)) < 0.5).astype(np.int64)
        v = rng.integers(1, hi, (n, tx))
        v[rng.random((n, tx)) < 0.1] = 0
    elif kind == "sparse":      # almost all state 0 without a finite value, a few far candidates
        st = (rng.random((n, tx)) < 0.003).astype(np.int64)
        v = np.where(rng.random((n, tx)) < 0.01, rng.integers(1, hi, (n, tx)), 0)
    elif kind == "empty":
        st = np.zeros((n, tx), np.int64)
        v = np.zeros((n, tx), np.int64)
    elif kind == "full":
        st = np.ones((n, tx), np.int64)
        v = np.zeros((n, tx), np.int64)
    elif kind == "constant":    # a solid block: every parabola is on the hull
        st = np.ones((n, tx), np.int64)
        st[: n // 7] = 0
        v = np.full((n, tx), min(hi - 1, 57), np.int64)
    elif kind == "runs":        # long same-state runs with smooth values
        st = ((np.arange(n)[:, None] // rng.integers(5, 90, tx)[None, :]) % 2).astype(np.int64)
        v = (np.abs(np.sin(np.arange(n)[:, None] * 0.07 + np.arange(tx)[None, :])) * (hi - 2) + 1).astype(np.int64)
    else:                       # one finite candidate per column
        st = np.zeros((n, tx), np.int64)
        v = np.zeros((n, tx), np.int64)
        for c in range(tx):
            v[rng.integers(0, n), c] = rng.integers(1, hi)
    return st, v


@pytest.mark.parametrize("dtype", [np.uint16, np.uint32])
@pytest.mark.parametrize("kind", CASES)
@pytest.mark.parametrize("n", [1, 31, 32, 33, 100, 257, 1024])
def test_hull_matches_brute_force(hull, dtype, kind, n):
    rng = np.random.default_rng(hash((kind, n, dtype.__name__)) & 0xFFFF)
    tx = 4
    st, v = gen(kind, n, tx, dtype, rng)
    run_case(hull, st, v, dtype)
    run_case(hull, st, v, dtype, sb=16)
