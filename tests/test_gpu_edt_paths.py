"""The mask EDT's three line-pass paths give the same floats as the oracle.

The y and z passes pick, per tile, the windowed search (every cell's own value
small), the lower-envelope path (csrc/hull.cuh; cells with no other-state
cell on their lower-dimension lines, e.g. sparse or empty volumes) or, for
the uint32 z pass, the block-pruned search (cells far from the other state in
their plane).  DOL_TUNE_EDT_HULL forces them: 1 = windowed search only, 2 =
envelope only, 101 = the pruned search for every z tile (windowed y), 102 =
the automatic choice without the pruned search, 0 = the automatic choice.  Every
setting must reproduce the reference's Felzenszwalb bit for bit, in all three
output forms, on dense, sparse, empty and full inputs, for lines of one or
several TMA boxes and both volume layouts (w a multiple of 8 or not).
"""
import hashlib
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
HULL = 10   # DOL_TUNE_EDT_HULL
HERE = os.path.dirname(os.path.abspath(__file__))


def _set_hull(L, v):
    for k in range(15):
        L.dol_tune_set(HULL, 1 << k, v)


@pytest.fixture
def hull_mode(dol):
    L = dol.lib()
    yield lambda v: _set_hull(L, v)
    _set_hull(L, 0)


def same_float(a, b):
    a, b = np.asarray(a, np.float32), np.asarray(b, np.float32)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def _case(O, rng, dims, kind):
    shape = tuple(reversed(dims))
    if kind == "points":
        b = rng.random(shape) < 3.0 / np.prod(shape) ** 0.5
    elif kind == "empty":
        b = np.zeros(shape, bool)
    elif kind == "full":
        b = np.ones(shape, bool)
    elif kind == "blocks":   # solid boxes: long runs with the same own value
        b = np.zeros(shape, bool)
        for _ in range(3):
            lo = [rng.integers(0, s) for s in shape]
            hi = [min(s, l + rng.integers(1, max(2, s // 2 + 1))) for l, s in zip(lo, shape)]
            b[tuple(slice(l, h) for l, h in zip(lo, hi))] = True
    else:
        b = rng.random(shape) < float(kind)
    return O.bool_to_mask(b)


DIMS = [(64, 64), (100, 37), (333, 129), (24, 20, 16), (33, 6, 5), (40, 70, 9), (64, 300, 20), (48, 40, 600),
        (16, 1030, 3)]
KINDS = ["points", "empty", "full", "blocks", "0.003", "0.3"]


@pytest.mark.parametrize("mode", [1, 2, 101, 102, 0])
@pytest.mark.parametrize("dims", DIMS)
def test_edt_paths_match_oracle(dol, O, cuda, hull_mode, dims, mode):
    torch = cuda
    hull_mode(mode)
    rng = np.random.default_rng(sum(dims) * 7 + mode)
    big = np.float32(np.finfo(np.float32).max)
    for kind in KINDS:
        m = _case(O, rng, dims, kind)
        md = torch.from_numpy(m.view(np.int32)).cuda()
        b = O.mask_to_bool(m, dims)
        want_sq = O.felzenszwalb(np.where(b, np.float32(0), big).astype(np.float32), dims)
        same_float(dol.edt_mask(md, dims, dol.EDT_SQUARED).cpu().numpy(), want_sq)
        same_float(dol.edt_mask(md, dims, dol.EDT_DIST).cpu().numpy(), np.sqrt(want_sq))
        same_float(dol.edt_mask(md, dims, dol.EDT_SIGNED).cpu().numpy(), O.sdf_signed_felzenszwalb(m, dims))


def test_edt_sparse_1024_against_reference_digests(dol, O, cuda):
    """1024^3 of 2000 points (BitMaskAddPoints, seed 1) and 1024^3 of none:
    the signed SDF's SHA-256 equals the reference's."""
    with open(os.path.join(HERE, "golden", "golden_digests.json")) as f:
        dig = json.load(f)
    if "s3_points2000_felz_signed" not in dig:
        pytest.skip("sparse digests not generated")
    torch = cuda
    n = 1024
    dims = (n, n, n)
    m = dol.add_points(np.zeros(dol.mask_words(*dims), np.uint32), dims, 2000, 1)
    assert hashlib.sha256(m.tobytes()).hexdigest() == dig["s3_points2000_mask"]
    for key, mask in (("s3_points2000_felz_signed", m), ("s3_empty_felz_signed", np.zeros_like(m))):
        md = torch.from_numpy(mask.view(np.int32)).cuda()
        sdf = dol.edt_mask(md, dims, dol.EDT_SIGNED)
        dol.sync()
        assert hashlib.sha256(sdf.cpu().numpy().tobytes()).hexdigest() == dig[key], key
        del sdf, md
        torch.cuda.empty_cache()
