"""Parity at the benchmarked sizes.

The library's outputs on the two benchmarked volumes against SHA-256 digests
of the reference's own outputs on the same masks (tests/golden/gen_golden.py
--full, run next to the reference checkout):

* 256^3, 32 boxes + 32 spheres (sides / radii 4-40, seed 7): border init,
  Danielsson / FastSweep / JumpFlood with cw = 2, signed Felzenszwalb SDF;
* 1024^3 value noise (lattice 16, seed 3): signed Felzenszwalb SDF (the
  headline workload, 4 GiB of f32) and signed Danielsson deltas (6 GiB).

The masks come from the library's device generators; their digests equal the
host generator's, which produced the golden inputs.
"""
import ctypes as C
import hashlib
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def dig():
    with open(os.path.join(HERE, "golden", "golden_digests.json")) as f:
        return json.load(f)


def sha(t):
    return hashlib.sha256(np.ascontiguousarray(t.cpu().numpy()).tobytes()).hexdigest()


def test_shapes_256_all_methods(dol, cuda, dig):
    n = 256
    dims = (n, n, n)
    L = dol.lib()
    md = cuda.empty(dol.mask_words(*dims), dtype=cuda.int32, device="cuda")
    dol.check(L.dol_gen_shapes_3d(n, n, n, 32, 32, 4, 40, C.c_uint32(7), C.c_void_p(md.data_ptr()), None))
    assert sha(md) == dig["c2_mask"]
    bor = dol.init_border(md, dims)
    assert sha(bor) == dig["c2_border"]
    for meth in ("danielsson", "fastsweep", "jumpflood"):
        got = dol.propagate(meth, bor.clone(), dims, 2)
        dol.sync()
        assert sha(got) == dig[f"c2_{meth}_cw2"], meth
    sdf = dol.edt_mask(md, dims, dol.EDT_SIGNED)
    dol.sync()
    assert sha(sdf) == dig["c2_felz_signed"]


def test_noise_1024_felzenszwalb_and_danielsson(dol, cuda, dig):
    n = 1024
    dims = (n, n, n)
    L = dol.lib()
    md = cuda.empty(dol.mask_words(*dims), dtype=cuda.int32, device="cuda")
    dol.check(L.dol_gen_value_noise_3d(n, n, n, 16, C.c_uint32(3), C.c_void_p(md.data_ptr()), None))
    assert sha(md) == dig["c3_mask"]
    sdf = dol.edt_mask(md, dims, dol.EDT_SIGNED)
    dol.sync()
    assert sha(sdf) == dig["c3_felz_signed"]
    del sdf
    dl = dol.init_border(md, dims)
    dol.danielsson(dl, dims, 2)
    dol.sync()
    assert sha(dl) == dig["c3_danielsson_cw2"]
    del dl
    cuda.cuda.empty_cache()
