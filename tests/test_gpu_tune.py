"""The launch-configuration table never changes results: every candidate value
of every family gives bit-identical output, and dol_autotune picks one of the
candidates and leaves results unchanged."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DAN2, DAN3, FS2, FS3, JFA2, JFA3, BATCH, EDT = range(8)


def _mask(O, dims, p, seed):
    rng = np.random.default_rng(seed)
    return O.bool_to_mask(rng.random(tuple(reversed(dims))) < p)


@pytest.mark.parametrize("kind,method,dims,values", [
    (DAN2, "danielsson", (300, 40), [1, 2, 4, 8, 32]),
    (FS2, "fastsweep", (300, 40), [1, 2, 4, 8, 32]),
    (DAN3, "danielsson", (70, 12, 9), [1, 2, 4, 8, 32]),
    (FS3, "fastsweep", (70, 12, 9), [1, 2, 4, 8, -1, -2, -4, -8]),
    (JFA2, "jumpflood", (300, 40), [2, 4, 8, 16]),
    (JFA3, "jumpflood", (70, 12, 9), [2, 4, 8, 16, -2, -4, -8, -16]),
    (JFA3, "jumpflood", (40, 33, 70), [8, -8]),
])
def test_every_candidate_gives_the_same_deltas(dol, O, cuda, kind, method, dims, values):
    torch = cuda
    L = dol.lib()
    m = _mask(O, dims, 0.05, kind)
    md = torch.from_numpy(m.view(np.int32)).cuda()
    want = O.propagate(method, O.border_init(m, dims), dims, 2)
    try:
        for v in values:
            L.dol_tune_set(kind, dims[0], v)
            got = dol.propagate(method, dol.init_border(md, dims), dims, 2)
            dol.sync()
            np.testing.assert_array_equal(got.cpu().numpy(), want, err_msg=f"value {v}")
    finally:
        L.dol_tune_set(kind, dims[0], 0)


def test_edt_threads_do_not_change_results(dol, O, cuda):
    torch = cuda
    L = dol.lib()
    dims = (64, 40, 48)
    m = _mask(O, dims, 0.3, 3)
    md = torch.from_numpy(m.view(np.int32)).cuda()
    want = O.sdf_signed_felzenszwalb(m, dims)
    try:
        for v in (256, 512):
            L.dol_tune_set(EDT, dims[0], v)
            got = dol.edt_mask(md, dims, dol.EDT_SIGNED).cpu().numpy()
            np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32))
    finally:
        L.dol_tune_set(EDT, dims[0], 0)


@pytest.mark.parametrize("kind,dims,values", [
    (DAN2, (512, 512, 1), {1, 2, 4, 8, 32}), (FS3, (128, 64, 32), {1, 2, 4, -1, -2, -4}),
    (JFA3, (128, 128, 128), {2, 4, 8, 16, -2, -4, -8, -16}),
    (EDT, (256, 256, 256), {256, 512}), (BATCH, (1024, 1, 1), {4, 8})])
def test_autotune_picks_a_candidate(dol, cuda, kind, dims, values):
    L = dol.lib()
    st = L.dol_autotune(kind, *dims, None)
    assert st == dol.OK, L.dol_last_error()
    v = L.dol_tune_get(kind, dims[0])
    assert v in values
    L.dol_tune_set(kind, dims[0], 0)
