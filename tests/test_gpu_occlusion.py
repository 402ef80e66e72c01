"""GPU occlusion sweeps against the CPU oracle and the reference build.

InitDirWFromBitMask and the quadrant / octant sweeps (in place, and the 3D
in/out form) through the C ABI must reproduce the reference bit for bit: the
GPU keeps the reference's serial float chain along each row, with every add
and multiply rounded on its own.  The oracle's restatement is pinned to the
reference in test_oracle_pin.py; here the reference build is compared
directly as well when it is present.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SHAPES = [(1, 1), (1, 9), (9, 1), (31, 7), (32, 8), (33, 13), (100, 37), (257, 19), (1025, 6), (2050, 3), (4096, 2),
          (65, 70), (5000, 3),
          (1, 1, 1), (5, 1, 3), (1, 4, 3), (9, 7, 5), (33, 6, 5), (24, 20, 16), (40, 70, 9), (1100, 3, 2),
          (40, 35, 70), (70, 33, 40), (4500, 2, 2)]
OCC = 11   # DOL_TUNE_OCCLUSION: 0 block wavefront, 1 one CTA per plane, n > 1 slices per 3D block (+1000: 32 rows)


@pytest.fixture
def engine(dol):
    """Sets the occlusion engine for every row length; puts the default back afterwards."""
    L = dol.lib()

    def put(v):
        for b in range(16):
            L.dol_tune_set(OCC, 1 << b, v)
    yield put
    put(0)


def same(a, b):
    np.testing.assert_array_equal(np.asarray(a, np.float32).view(np.uint32), np.asarray(b, np.float32).view(np.uint32))


def _engines(dims):
    """The default, one CTA per plane where the rows allow it, 3D blocks of 8 slices and of 32 rows x 64 slices."""
    e = [0]
    if dims[0] <= 4096:
        e.append(1)
    if len(dims) == 3:
        e += [8, 1064]
    return e


CASES = [(d, e) for d in SHAPES for e in _engines(d)]


@pytest.mark.parametrize("dims,eng", CASES, ids=[f"{'x'.join(map(str, d))}-e{e}" for d, e in CASES])
def test_occlusion_matches_oracle(dol, O, cuda, engine, dims, eng):
    torch = cuda
    engine(eng)
    rng = np.random.default_rng(sum(dims) + 5)
    for p in (0.0, 0.05, 0.4, 1.0):
        m = O.bool_to_mask(rng.random(tuple(reversed(dims))) < p)
        md = torch.from_numpy(m.view(np.int32)).cuda()
        dw = dol.init_dirw(md, dims)
        want0 = O.init_dirw(m, dims)
        same(dw.cpu().numpy(), want0)
        got = dol.occlusion_sweep(dw.clone(), dims).cpu().numpy()
        same(got, O.occlusion_sweep(want0, dims))
        if O.ref() is not None and np.prod(dims) <= 70000:
            same(got, O.occlusion_sweep(want0, dims, use_ref=True))
        if len(dims) == 3:
            prior = rng.random(want0.shape).astype(np.float32)
            out = torch.from_numpy(prior).cuda()
            got = dol.occlusion_sweep_io(dw, out, dims).cpu().numpy()
            same(got, O.occlusion_sweep_io(want0, prior, dims))


@pytest.mark.parametrize("dims", [(1024, 1024), (128, 128, 128)])
def test_occlusion_configuration_sizes(dol, O, cuda, dims):
    """The 2D default image (100 points, seed 1) and a 128^3 volume of value noise."""
    import ctypes as C
    torch = cuda
    if len(dims) == 2:
        m = dol.add_points(np.zeros(dol.mask_words(*dims), np.uint32), dims, 100, 1)
    else:
        m = np.zeros(dol.mask_words(*dims), np.uint32)
        dol.lib().dol_gen_value_noise_3d_host(*dims, 16, C.c_uint32(3), m.ctypes.data_as(C.c_void_p))
    md = torch.from_numpy(m.view(np.int32)).cuda()
    got = dol.occlusion_sweep(dol.init_dirw(md, dims), dims).cpu().numpy()
    want = O.occlusion_sweep(O.init_dirw(m, dims), dims, use_ref=O.ref() is not None)
    same(got, want)


@pytest.mark.parametrize("eng", [0, 1])
@pytest.mark.parametrize("dims", [(1024, 1024), (128, 128, 128)])
def test_occlusion_engines_agree_at_configuration_sizes(dol, O, cuda, engine, dims, eng):
    """Both engines on the configuration sizes, through the in-place and (3D) in/out forms."""
    import ctypes as C
    torch = cuda
    rng = np.random.default_rng(11)
    m = O.bool_to_mask(rng.random(tuple(reversed(dims))) < 0.05)
    md = torch.from_numpy(m.view(np.int32)).cuda()
    engine(eng)
    dw = dol.init_dirw(md, dims)
    got = dol.occlusion_sweep(dw.clone(), dims).cpu().numpy()
    want0 = O.init_dirw(m, dims)
    same(got, O.occlusion_sweep(want0, dims))
    if len(dims) == 3:
        prior = rng.random(want0.shape).astype(np.float32)
        got = dol.occlusion_sweep_io(dw, torch.from_numpy(prior).cuda(), dims).cpu().numpy()
        same(got, O.occlusion_sweep_io(want0, prior, dims))


def test_occlusion_rejects_aliasing(dol, cuda):
    torch = cuda
    buf = torch.zeros(8 * 10 * 2 * 2, dtype=torch.float32, device="cuda")
    with pytest.raises(dol.DolError):
        dol.occlusion_sweep_io(buf, buf, (10, 2, 2))
