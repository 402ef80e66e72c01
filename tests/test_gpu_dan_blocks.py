"""Danielsson's block schedule (fixed-point iteration over blocks of rows)
against the oracle's serial Danielsson, bit for bit, for every rows-per-block
value, slices-per-block value and cells-per-thread engine, on masks of awkward shapes and densities,
signed (border init, cw = 2) and unsigned (cw = 1)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TUNE_DAN2, TUNE_DAN3, TUNE_ROWS, TUNE_SLICES = 0, 1, 8, 9
SERIAL = 65536


def dev(torch, a):
    a = np.ascontiguousarray(a)
    if a.dtype == np.uint32:
        a = a.view(np.int32)
    return torch.from_numpy(a).cuda()


def rand_mask(O, rng, dims, p):
    return O.bool_to_mask(rng.random(tuple(reversed(dims))) < p)


def blob_mask(O, rng, dims, n):
    """a few solid balls: long empty stretches, the slow case for the rounds"""
    grid = np.meshgrid(*[np.arange(k) for k in reversed(dims)], indexing="ij")
    b = np.zeros(tuple(reversed(dims)), bool)
    for _ in range(n):
        c = [rng.integers(0, k) for k in reversed(dims)]
        r = rng.integers(1, 1 + max(2, min(dims) // 4))
        b |= sum((g - ci) ** 2 for g, ci in zip(grid, c)) <= r * r
    return O.bool_to_mask(b)


@pytest.fixture
def tune(dol):
    L = dol.lib()
    touched = []

    def set_(kind, w, v):
        touched.append((kind, w))
        L.dol_tune_set(kind, w, v)
    yield set_
    for kind, w in touched:
        L.dol_tune_set(kind, w, 0)


def run(dol, cuda, O, m, dims, cw, signed):
    md = dev(cuda, m)
    dl = dol.init_border(md, dims) if signed else dol.init_deltas(md, dims)
    dol.danielsson(dl, dims, cw)
    dol.sync()
    ini = O.border_init(m, dims) if signed else O.init_deltas(m, dims)
    return dl.cpu().numpy(), O.propagate("danielsson", ini, dims, cw)


SHAPES3 = [(37, 29, 23), (64, 17, 40), (5, 80, 9), (130, 33, 12), (1, 20, 30), (40, 1, 25)]
SHAPES2 = [(200, 150), (1024, 77), (33, 500), (1, 300), (300, 1), (517, 260)]


@pytest.mark.parametrize("slices", [1, 2, 5, 1000])
@pytest.mark.parametrize("rows", [1, 3, 8, 64])
@pytest.mark.parametrize("dims", SHAPES3)
def test_blocks_3d(dol, O, cuda, tune, dims, rows, slices):
    rng = np.random.default_rng(sum(dims) + rows + slices)
    tune(TUNE_ROWS, dims[0], rows)
    tune(TUNE_SLICES, dims[0], slices)
    for i, m in enumerate([rand_mask(O, rng, dims, 0.002), rand_mask(O, rng, dims, 0.3), blob_mask(O, rng, dims, 3),
                           rand_mask(O, rng, dims, 0.0)]):
        for cw, signed in ((2, True), (1, False)):
            got, want = run(dol, cuda, O, m, dims, cw, signed)
            np.testing.assert_array_equal(got, want, err_msg=f"mask {i} cw {cw}")


@pytest.mark.parametrize("rows", [1, 5, 8, 64])
@pytest.mark.parametrize("dims", SHAPES2)
def test_blocks_2d(dol, O, cuda, tune, dims, rows):
    rng = np.random.default_rng(sum(dims) + rows)
    tune(TUNE_ROWS, dims[0], rows)
    for i, m in enumerate([rand_mask(O, rng, dims, 0.0005), rand_mask(O, rng, dims, 0.2), blob_mask(O, rng, dims, 4)]):
        for cw, signed in ((2, True), (1, False)):
            got, want = run(dol, cuda, O, m, dims, cw, signed)
            np.testing.assert_array_equal(got, want, err_msg=f"mask {i} cw {cw}")


@pytest.mark.parametrize("cells_per_thread", [1, 2, 4, 8])
def test_blocks_engines(dol, O, cuda, tune, cells_per_thread):
    rng = np.random.default_rng(cells_per_thread)
    for dims, kind in (((700, 40, 20), TUNE_DAN3), ((1500, 90), TUNE_DAN2)):
        tune(TUNE_ROWS, dims[0], 8)
        tune(kind, dims[0], cells_per_thread)
        m = blob_mask(O, rng, dims, 5)
        got, want = run(dol, cuda, O, m, dims, 2, True)
        np.testing.assert_array_equal(got, want)


def test_blocks_match_serial_engine(dol, O, cuda, tune):
    """default schedule vs the serial single-CTA engine on a 96^3 shape volume"""
    import ctypes as C
    L = dol.lib()
    n = 96
    dims = (n, n, n)
    md = cuda.empty(dol.mask_words(*dims), dtype=cuda.int32, device="cuda")
    dol.check(L.dol_gen_shapes_3d(n, n, n, 12, 12, 3, 20, C.c_uint32(5), C.c_void_p(md.data_ptr()), None))
    base = dol.init_border(md, dims)
    a = base.clone()
    dol.danielsson(a, dims, 2)
    tune(TUNE_ROWS, n, SERIAL)
    b = base.clone()
    dol.danielsson(b, dims, 2)
    dol.sync()
    assert cuda.equal(a, b)
    want = O.propagate("danielsson", O.border_init(md.cpu().numpy().view(np.uint32), dims), dims, 2)
    np.testing.assert_array_equal(a.cpu().numpy(), want)


# ---- workspace: the caller's, the library's, or none (serial engine, reported) ----------------

ENGINE_BLOCKS, ENGINE_SERIAL = 1, 2


@pytest.mark.parametrize("dims", [(300, 257), (96, 80, 40)])
def test_danielsson_workspace_paths_agree_and_fallback_is_reported(dol, O, cuda, dims):
    """The block schedule on the caller's workspace (the _ws entries), on the
    library's own allocation, and -- with the library's allocations capped
    below the workspace size -- the serial engine: identical deltas, equal to
    the oracle, and the fallback shows in dol_last_engine() / dol_last_error()."""
    import ctypes as C
    torch = cuda
    L = dol.lib()
    rng = np.random.default_rng(sum(dims) + 77)
    m = rand_mask(O, rng, dims, 0.02)
    md = dev(torch, m)
    bor = dol.init_border(md, dims)
    want = O.propagate("danielsson", O.border_init(m, dims), dims, 2)
    wd = dims + (1,) if len(dims) == 2 else dims
    need = L.dol_danielsson_workspace_size(*wd)
    assert need > 0
    sp = C.c_void_p(torch.cuda.current_stream().cuda_stream)

    def run(fn, *extra):
        work = bor.clone()
        st = fn(*dims, C.c_void_p(work.data_ptr()), 2, *extra, sp)
        assert st == dol.OK, L.dol_last_error()
        engine = L.dol_last_engine()
        note = L.dol_last_error()
        dol.sync()
        np.testing.assert_array_equal(work.cpu().numpy(), want)
        return engine, note

    plain, ws_fn = ((L.dol_danielsson_2d, L.dol_danielsson_2d_ws) if len(dims) == 2
                    else (L.dol_danielsson_3d, L.dol_danielsson_3d_ws))
    ws = torch.empty(need, dtype=torch.uint8, device="cuda")
    assert run(ws_fn, C.c_void_p(ws.data_ptr()), C.c_size_t(need))[0] == ENGINE_BLOCKS
    assert run(plain)[0] == ENGINE_BLOCKS
    L.dol_set_workspace_limit(C.c_size_t(need // 2))
    try:
        engine, note = run(plain)
        assert engine == ENGINE_SERIAL and b"serial engine" in note and b"dol_set_workspace_limit" in note
        # the caller's workspace is not subject to the cap
        assert run(ws_fn, C.c_void_p(ws.data_ptr()), C.c_size_t(need))[0] == ENGINE_BLOCKS
    finally:
        L.dol_set_workspace_limit(C.c_size_t(0))
    # a caller's workspace that is too small is an error, not a silent fallback
    work = bor.clone()
    st = ws_fn(*dims, C.c_void_p(work.data_ptr()), 2, C.c_void_p(ws.data_ptr()), C.c_size_t(need - 1), sp)
    assert st == dol.ERR_INVALID_ARG and b"workspace too small" in L.dol_last_error()
