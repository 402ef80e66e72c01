"""GPU parity: every entry point of the CUDA library against the CPU oracle on
the same inputs, through the C ABI.  Integer outputs (masks, deltas) must be
bit-exact; float outputs are compared bit-for-bit as well, because every float
the reference produces on this path is a correctly rounded function of an
integer (sqrtf of an exact squared length, or the exact squared EDT)."""
import hashlib
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


def dev(torch, a):
    a = np.ascontiguousarray(a)
    if a.dtype == np.uint32:
        a = a.view(np.int32)
    return torch.from_numpy(a).cuda()


def host(t):
    a = t.cpu().numpy()
    return a.view(np.uint32) if a.dtype == np.int32 else a


def same_float(a, b):
    """bitwise equal, treating any NaN as equal to any NaN"""
    a, b = np.asarray(a, np.float32), np.asarray(b, np.float32)
    na, nb = np.isnan(a), np.isnan(b)
    assert np.array_equal(na, nb)
    assert np.array_equal(a.view(np.uint32)[~na], b.view(np.uint32)[~nb])


def rand_mask(O, rng, dims, p):
    return O.bool_to_mask(rng.random(tuple(reversed(dims))) < p)


SHAPES2 = [(1, 1), (1, 9), (9, 1), (31, 7), (32, 8), (33, 13), (64, 64), (100, 37), (257, 19), (1000, 5)]
SHAPES3 = [(1, 1, 1), (5, 1, 1), (1, 4, 3), (9, 7, 5), (32, 3, 4), (33, 6, 5), (40, 1, 6), (24, 20, 16)]
PS = (0.0, 0.01, 0.2, 0.6, 1.0)


@pytest.mark.parametrize("dims", SHAPES2 + SHAPES3)
def test_init_and_border(dol, O, cuda, dims):
    rng = np.random.default_rng(sum(dims))
    for p in PS:
        m = rand_mask(O, rng, dims, p)
        md = dev(cuda, m)
        for inv in (False, True):
            np.testing.assert_array_equal(host(dol.init_deltas(md, dims, inv)), O.init_deltas(m, dims, inv))
        np.testing.assert_array_equal(host(dol.init_border(md, dims)), O.border_init(m, dims), err_msg=f"p={p}")
        if len(dims) == 2:
            same_float(host(dol.init_distances(md, dims)), O.init_distances(m, dims))


@pytest.mark.parametrize("method", ["danielsson", "fastsweep", "jumpflood"])
@pytest.mark.parametrize("dims", SHAPES2 + SHAPES3)
def test_delta_methods(dol, O, cuda, dims, method):
    rng = np.random.default_rng(sum(dims) + len(method))
    for p in PS:
        m = rand_mask(O, rng, dims, p)
        md = dev(cuda, m)
        for cw in (1, 2):
            start = O.init_deltas(m, dims) if cw == 1 else O.border_init(m, dims)
            want = O.propagate(method, start, dims, cw)
            got = dol.propagate(method, dev(cuda, start), dims, cw)
            dol.sync()
            np.testing.assert_array_equal(host(got), want, err_msg=f"{method} cw{cw} p{p} dims{dims}")


@pytest.mark.parametrize("method", ["danielsson", "fastsweep", "jumpflood"])
@pytest.mark.parametrize("dims", [(4096, 6), (2049, 9), (2048, 3, 3), (1025, 2, 4)])
def test_delta_methods_widest_rows(dol, O, cuda, dims, method):
    """Rows at and around the sweep engines' limits (4096 cells in 2D; 2048 for
    3D FastSweep), past the block schedule's 2048, odd lengths."""
    rng = np.random.default_rng(sum(dims) + len(method) + 1)
    for p in (0.001, 0.3):
        m = rand_mask(O, rng, dims, p)
        for cw in (1, 2):
            start = O.init_deltas(m, dims) if cw == 1 else O.border_init(m, dims)
            want = O.propagate(method, start, dims, cw)
            got = dol.propagate(method, dev(cuda, start), dims, cw)
            dol.sync()
            np.testing.assert_array_equal(host(got), want, err_msg=f"{method} cw{cw} p{p} dims{dims}")


@pytest.mark.parametrize("dims", [(1024, 1024)])
def test_config1_against_reference_digests(dol, O, cuda, dims):
    with open(os.path.join(HERE, "golden", "golden_digests.json")) as f:
        dig = json.load(f)
    m = dol.add_points(np.zeros(dol.mask_words(*dims), np.uint32), dims, 100, 1)
    assert hashlib.sha256(m.tobytes()).hexdigest() == dig["c1_mask"]
    md = dev(cuda, m)
    for method in ("danielsson", "fastsweep", "jumpflood"):
        got = host(dol.propagate(method, dol.init_deltas(md, dims), dims, 1))
        assert hashlib.sha256(got.tobytes()).hexdigest() == dig[f"c1_{method}_cw1"], method
        got = host(dol.propagate(method, dol.init_border(md, dims), dims, 2))
        assert hashlib.sha256(got.tobytes()).hexdigest() == dig[f"c1_{method}_cw2"], method
    sq = host(dol.edt_mask(md, dims, dol.EDT_SQUARED))
    assert hashlib.sha256(sq.tobytes()).hexdigest() == dig["c1_felz"]


def test_config1_error_histogram_vs_bruteforce(dol, O, cuda):
    """The 1024^2 image with 100 points (seed 1): the GPU Danielsson's error
    histogram against BruteForce (the tool's PrintError measure) equals the
    reference CPU Danielsson's, and its maximum error is below one cell (the
    tool's pass criterion)."""
    dims = (1024, 1024)
    m = dol.add_points(np.zeros(dol.mask_words(*dims), np.uint32), dims, 100, 1)
    ini = O.init_deltas(m, dims)
    got = host(dol.propagate("danielsson", dol.init_deltas(dev(cuda, m), dims), dims, 1))
    bf = O.propagate("bruteforce", ini, dims, 1)
    want = O.propagate("danielsson", ini, dims, 1)
    h_gpu, max_gpu = O.error_histogram(got, bf, dims)
    h_cpu, max_cpu = O.error_histogram(want, bf, dims)
    np.testing.assert_array_equal(h_gpu, h_cpu)
    assert max_gpu == max_cpu < 1.0
    assert h_gpu.sum() == dims[0] * dims[1]


def test_volume64_against_reference_digests(dol, O, cuda):
    with open(os.path.join(HERE, "golden", "golden_digests.json")) as f:
        dig = json.load(f)
    dims = (64, 64, 64)
    m = dol.add_points(dol.add_block(np.zeros(dol.mask_words(*dims), np.uint32), dims, 6), dims, 200, 12345)
    assert hashlib.sha256(m.tobytes()).hexdigest() == dig["v64_mask"]
    md = dev(cuda, m)
    bor = dol.init_border(md, dims)
    assert hashlib.sha256(host(bor).tobytes()).hexdigest() == dig["v64_border"]
    for method in ("danielsson", "fastsweep", "jumpflood"):
        got = host(dol.propagate(method, dol.init_border(md, dims), dims, 2))
        dol.sync()
        assert hashlib.sha256(got.tobytes()).hexdigest() == dig[f"v64_{method}_cw2"], method
        got = host(dol.propagate(method, dol.init_deltas(md, dims), dims, 1))
        assert hashlib.sha256(got.tobytes()).hexdigest() == dig[f"v64_{method}_cw1"], method


@pytest.mark.parametrize("dims", SHAPES2 + SHAPES3 + [(300, 200), (70, 60, 50)])
def test_edt_mask_forms(dol, O, cuda, dims):
    rng = np.random.default_rng(sum(dims) + 99)
    big = np.float32(np.finfo(np.float32).max)
    for p in (0.0, 0.003, 0.05, 0.5, 1.0):
        m = rand_mask(O, rng, dims, p)
        md = dev(cuda, m)
        b = O.mask_to_bool(m, dims)
        want_sq = O.felzenszwalb(np.where(b, np.float32(0), big).astype(np.float32), dims)
        same_float(host(dol.edt_mask(md, dims, dol.EDT_SQUARED)), want_sq)
        same_float(host(dol.edt_mask(md, dims, dol.EDT_DIST)), np.sqrt(want_sq))
        same_float(host(dol.edt_mask(md, dims, dol.EDT_SIGNED)), O.sdf_signed_felzenszwalb(m, dims))


def test_edt_every_small_squared_distance(dol, O, cuda):
    """One set voxel at the origin of a 64^3 volume: the EDT takes every value
    x^2 + y^2 + z^2 below 4096 -- every squared distance a volume can give in
    that range -- so the distances cover every square root the library takes
    from its table; each must equal the correctly rounded sqrt of the integer."""
    n = 64
    b = np.zeros((n, n, n), dtype=bool)
    b[0, 0, 0] = True
    md = dev(cuda, O.bool_to_mask(b))
    z, y, x = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    sq = (x * x + y * y + z * z).astype(np.int64)
    want = np.sqrt(sq.astype(np.float32))
    assert len(np.unique(sq[sq < 4096])) > 3000
    same_float(host(dol.edt_mask(md, (n, n, n), dol.EDT_DIST)), want)
    same_float(host(dol.edt_mask(md, (n, n, n), dol.EDT_SQUARED)), sq.astype(np.float32))
    signed = host(dol.edt_mask(md, (n, n, n), dol.EDT_SIGNED))
    same_float(signed[1:, :, :], want[1:, :, :])


@pytest.mark.parametrize("method", ["danielsson", "fastsweep", "jumpflood"])
@pytest.mark.parametrize("dims", [(1, 1), (31, 7), (64, 64), (100, 37), (257, 19), (1, 4, 3), (9, 7, 5), (33, 6, 5),
                                  (24, 20, 16)])
def test_sdf_two_pass(dol, O, cuda, dims, method):
    """The tool's -S field: exterior and interior deltas bit-exact, Dist(ext) - Dist(int) identical floats."""
    rng = np.random.default_rng(sum(dims) + len(method) + 5)
    for p in PS:
        m = rand_mask(O, rng, dims, p)
        de, di, df = dol.sdf_two_pass(dev(cuda, m), dims, method)
        dol.sync()
        we, wi, wd = O.sdf_two_pass(m, dims, method)
        np.testing.assert_array_equal(host(de), we, err_msg=f"exterior {method} p{p}")
        np.testing.assert_array_equal(host(di), wi, err_msg=f"interior {method} p{p}")
        same_float(host(df), wd)
        _, _, only = dol.sdf_two_pass(dev(cuda, m), dims, method, want_deltas=False)
        dol.sync()
        same_float(host(only), wd)


@pytest.mark.parametrize("dims", [(2, 1), (2, 9), (3, 1), (31, 7), (64, 64), (100, 37), (257, 19), (1000, 5),
                                  (4096, 3), (33, 300), (2, 100), (5, 2000), (100, 129), (300, 257), (1024, 1024)])
def test_chamfer(dol, O, cuda, dims):
    """Chamfer 3-4 on int16 and int32 fields against the oracle, bit for bit: the
    tool's init (INT16_MAX - 16), masks of every density, and arbitrary values
    (int16: the whole range; int32: up to INT32_MAX - 4, where the reference's
    own sums stop wrapping)."""
    import torch
    rng = np.random.default_rng(sum(dims) + 41)
    for p in PS:
        m = rand_mask(O, rng, dims, p)
        md = dev(cuda, m)
        for dt, tdt, mx in ((np.int16, torch.int16, 32767 - 16), (np.int32, torch.int32, 2**31 - 1 - 16)):
            f = dol.init_distances_int(md, dims, dtype=str(tdt), max_d=mx)
            want_f = O.init_distances_int(m, dims, dt, mx)
            np.testing.assert_array_equal(f.cpu().numpy(), want_f)
            assert dol.chamfer(f, dims) == 3
            dol.sync()
            np.testing.assert_array_equal(f.cpu().numpy(), O.chamfer(want_f, dims)[0], err_msg=f"{dt} p{p}")
    shape = tuple(reversed(dims))
    for dt, lo, hi in ((np.int16, -32768, 32767), (np.int32, -2**31, 2**31 - 1 - 4)):
        f = rng.integers(lo, hi, size=shape, dtype=np.int64, endpoint=True).astype(dt)
        t = torch.from_numpy(f.copy()).cuda()
        dol.chamfer(t, dims)
        dol.sync()
        np.testing.assert_array_equal(t.cpu().numpy(), O.chamfer(f, dims)[0], err_msg=f"arbitrary {dt}")


def test_chamfer_rejects_bad_widths(dol, cuda):
    import torch
    for w in (1, 4097):
        t = torch.zeros((3, w), dtype=torch.int16, device="cuda")
        with pytest.raises(dol.DolError):
            dol.chamfer(t, (w, 3))


@pytest.mark.parametrize("dims", [(24, 20, 16), (40, 70, 9), (33, 100, 20), (64, 130, 3)])
def test_edt_mask_host_chunked(dol, O, cuda, dims):
    """dol_edt_mask_3d_host: host buffers, the last pass in y chunks with the copy
    back overlapping it; same floats as the oracle in every form."""
    rng = np.random.default_rng(sum(dims) + 3)
    big = np.float32(np.finfo(np.float32).max)
    for p in (0.0, 0.02, 0.4, 1.0):
        m = rand_mask(O, rng, dims, p)
        b = O.mask_to_bool(m, dims)
        want_sq = O.felzenszwalb(np.where(b, np.float32(0), big).astype(np.float32), dims)
        same_float(dol.edt_mask_host(m, dims, dol.EDT_SQUARED), want_sq)
        same_float(dol.edt_mask_host(m, dims, dol.EDT_SIGNED), O.sdf_signed_felzenszwalb(m, dims))


@pytest.mark.parametrize("dims", [(8, 1000, 3), (16, 300, 37), (24, 5, 777), (8, 2049, 2), (40, 3, 1029),
                                  (2000, 8), (64, 1027), (4096, 5), (8, 4096, 2)])
def test_edt_mask_long_lines(dol, O, cuda, dims):
    """Long y / z lines: several TMA boxes, lengths off the 4 / 32 grid, runs
    longer than a word, searches that reach the line ends."""
    rng = np.random.default_rng(sum(dims) + 7)
    big = np.float32(np.finfo(np.float32).max)
    for p in (0.0, 0.0005, 0.01, 0.3, 0.97, 1.0):
        m = rand_mask(O, rng, dims, p)
        md = dev(cuda, m)
        b = O.mask_to_bool(m, dims)
        want_sq = O.felzenszwalb(np.where(b, np.float32(0), big).astype(np.float32), dims)
        same_float(host(dol.edt_mask(md, dims, dol.EDT_SQUARED)), want_sq)
        same_float(host(dol.edt_mask(md, dims, dol.EDT_SIGNED)), O.sdf_signed_felzenszwalb(m, dims))


@pytest.mark.parametrize("dims", [(16384, 4), (16384, 3, 2), (12345, 5), (5000, 3)])
def test_edt_mask_rows_beyond_float_exactness(dol, O, cuda, dims):
    """Rows longer than 4096 cells: the reference's float envelope is no longer
    exact there (its q*q passes 2^24; an all-set 5000 x 3 image already gets
    nonzero distances), so the check is the exact EDT, which the library keeps
    computing in integers (16384-cell rows also take the x pass's chunk carries)."""
    rng = np.random.default_rng(sum(dims) + 11)
    big = np.float32(np.finfo(np.float32).max)
    for p in (0.0, 0.0005, 0.01, 0.3, 1.0):
        m = rand_mask(O, rng, dims, p)
        md = dev(cuda, m)
        ex = O.edt_exact_thin(m, dims)
        want_sq = np.where(ex < 0, big, ex.astype(np.float32)).astype(np.float32)
        same_float(host(dol.edt_mask(md, dims, dol.EDT_SQUARED)), want_sq)
        same_float(host(dol.edt_mask(md, dims, dol.EDT_SIGNED)), O.sdf_signed_exact_thin(m, dims))


@pytest.mark.parametrize("dims", [(1, 1), (7, 1), (1, 7), (33, 17), (64, 48), (200, 130)])
def test_felzenszwalb_float_field(dol, O, cuda, dims):
    """DOL::Felzenszwalb on arbitrary floats, not just 0 / FLT_MAX."""
    rng = np.random.default_rng(sum(dims))
    w, h = dims
    big = np.float32(np.finfo(np.float32).max)
    for kind in range(3):
        if kind == 0:
            f = (rng.random((h, w)) * 50).astype(np.float32)
        elif kind == 1:
            f = np.where(rng.random((h, w)) < 0.1, (rng.random((h, w)) * 3).astype(np.float32), big)
        else:
            f = np.where(rng.random((h, w)) < 0.02, np.float32(0), big).astype(np.float32)
        want = O.felzenszwalb(f, dims)
        got = dol.felzenszwalb(dev(cuda, f.astype(np.float32)), dims)
        same_float(host(got), want)


@pytest.mark.parametrize("dims", SHAPES2 + SHAPES3)
def test_deltas_to_dist(dol, O, cuda, dims):
    rng = np.random.default_rng(sum(dims) + 3)
    m = rand_mask(O, rng, dims, 0.2)
    for cw, start in ((1, O.init_deltas(m, dims)), (2, O.border_init(m, dims))):
        dl = O.propagate("danielsson", start, dims, cw)
        for sign in (None, m):
            want = O.deltas_to_dist(dl, dims, cw, sign)
            got = dol.deltas_to_dist(dev(cuda, dl), dims, cw, None if sign is None else dev(cuda, sign))
            same_float(host(got), want)


@pytest.mark.parametrize("dims", [(1, 1), (33, 5), (100, 37), (64, 8, 5)])
def test_pack_bytemask(dol, O, cuda, dims):
    rng = np.random.default_rng(sum(dims))
    img = rng.integers(0, 256, size=tuple(reversed(dims)), dtype=np.uint8)
    for thr, lt in ((128, True), (128, False), (0, True), (255, False)):
        got = host(dol.pack_bytemask(dev(cuda, img), thr, lt))
        if len(dims) == 2:
            want = O.pack_bytes(img, thr, lt)
        else:
            want = O.pack_bytes(img.reshape(-1, dims[0]), thr, lt)
        np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("method", ["danielsson", "fastsweep", "jumpflood", "felzenszwalb"])
@pytest.mark.parametrize("dims", [(64, 48), (33, 20, 17)])
def test_sdf_pipeline_device_and_host(dol, O, cuda, dims, method):
    rng = np.random.default_rng(7)
    m = rand_mask(O, rng, dims, 0.3)
    if method == "felzenszwalb":
        want_dl, want_df = None, O.sdf_signed_felzenszwalb(m, dims)
    else:
        want_dl = O.propagate(method, O.border_init(m, dims), dims, 2)
        want_df = O.deltas_to_dist(want_dl, dims, 2, m)
    dl, df = dol.sdf(dev(cuda, m), dims, method)
    dol.sync()
    if want_dl is not None:
        np.testing.assert_array_equal(host(dl), want_dl)
    same_float(host(df), want_df)
    hdl, hdf = dol.sdf_host(m, dims, method)
    if want_dl is not None:
        np.testing.assert_array_equal(hdl, want_dl)
    same_float(hdf, want_df)


def test_word_boundary_single_seeds(dol, O, cuda):
    """A lone set cell at x = 30, 31, 32 exercises the cross-word write order
    of the border initialisation (the x = 31 case ends as (1, 0))."""
    for dims in [(64, 4), (96, 3), (64, 3, 3)]:
        for x in (0, 30, 31, 32, 33, 63):
            b = np.zeros(tuple(reversed(dims)), bool)
            if len(dims) == 2:
                b[1, x] = True
            else:
                b[1, 1, x] = True
            m = O.bool_to_mask(b)
            got = host(dol.init_border(dev(cuda, m), dims))
            np.testing.assert_array_equal(got, O.border_init(m, dims), err_msg=f"x={x} {dims}")


def test_rejects_bad_arguments(dol, cuda):
    import ctypes as C
    L = dol.lib()
    buf = cuda.zeros(64, dtype=cuda.int32, device="cuda")
    hostbuf = np.zeros(64, np.uint32)
    st = L.dol_init_border_2d(C.c_int(32), C.c_int(2), hostbuf.ctypes.data_as(C.c_void_p),
                              C.c_void_p(buf.data_ptr()), None)
    assert st == dol.ERR_INVALID_ARG
    st = L.dol_init_border_2d(C.c_int(0), C.c_int(2), C.c_void_p(buf.data_ptr()), C.c_void_p(buf.data_ptr()), None)
    assert st == dol.ERR_INVALID_ARG
    st = L.dol_danielsson_2d(C.c_int(5000), C.c_int(2), C.c_void_p(buf.data_ptr()), C.c_int(1), None)
    assert st == dol.ERR_UNSUPPORTED
    with pytest.raises(dol.DolError):
        dol.edt_mask(buf, (32, 2), form=7)
