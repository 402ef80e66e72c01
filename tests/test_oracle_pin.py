"""Pin the CPU oracle (oracle/dol_oracle.c) to the reference.

1. Against the committed golden vectors (tests/golden/), which were produced
   by the unmodified reference library (tests/golden/gen_golden.py).
2. Against the reference library itself (oracle/_ref), when it was built here,
   on randomised masks of awkward shapes, empty and full masks, and garbage in
   the row padding bits.
3. Against the reference's README images (images/*-sdf.png regenerated from
   data/*.png), which reproduce within +-1 grey level -- a weak check, run only
   where the reference checkout exists: the directory in DOL_REFERENCE_DIR, or
   the one oracle/Makefile recorded in oracle/_ref/ref_dir.txt when it built
   the reference.
"""
import hashlib
import json
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")


def _reference_dir():
    """The reference checkout: DOL_REFERENCE_DIR, else the directory the oracle
    recipe built oracle/_ref from; None when neither names an existing one."""
    d = os.environ.get("DOL_REFERENCE_DIR")
    if not d:
        rec = os.path.join(os.path.dirname(HERE), "oracle", "_ref", "ref_dir.txt")
        if os.path.exists(rec):
            with open(rec) as f:
                d = f.read().strip()
    return d if d and os.path.isdir(d) else None


REF_DIR = _reference_dir()


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.fixture(scope="module")
def small():
    return np.load(os.path.join(GOLD, "golden_small.npz"))


@pytest.fixture(scope="module")
def digests():
    with open(os.path.join(GOLD, "golden_digests.json")) as f:
        return json.load(f)


def _names(small):
    return sorted({k.rsplit("_mask", 1)[0] for k in small.files if k.endswith("_mask")})


def test_oracle_matches_golden_small(O, small):
    for name in _names(small):
        m = small[f"{name}_mask"]
        dims = tuple(int(x) for x in small[f"{name}_dims"])
        ini = O.init_deltas(m, dims)
        bor = O.border_init(m, dims)
        np.testing.assert_array_equal(ini, small[f"{name}_init"], err_msg=name)
        np.testing.assert_array_equal(bor, small[f"{name}_border"], err_msg=name)
        if f"{name}_init_inv" in small.files:
            np.testing.assert_array_equal(O.init_deltas(m, dims, True), small[f"{name}_init_inv"], err_msg=name)
        for meth in ("danielsson", "fastsweep", "jumpflood"):
            np.testing.assert_array_equal(O.propagate(meth, ini, dims, 1), small[f"{name}_{meth}_cw1"],
                                          err_msg=f"{name} {meth} cw1")
            np.testing.assert_array_equal(O.propagate(meth, bor, dims, 2), small[f"{name}_{meth}_cw2"],
                                          err_msg=f"{name} {meth} cw2")
        np.testing.assert_array_equal(O.propagate("bruteforce", ini, dims, 1), small[f"{name}_bruteforce_cw1"])
        if len(dims) == 2:
            np.testing.assert_array_equal(O.propagate("bruteforce", bor, dims, 2), small[f"{name}_bruteforce_cw2"])
            f = O.init_distances(m, dims)
            np.testing.assert_array_equal(O.felzenszwalb(f, dims), small[f"{name}_felz"])
        else:
            big = np.float32(np.finfo(np.float32).max)
            f = np.where(O.mask_to_bool(m, dims), np.float32(0), big).astype(np.float32)
            np.testing.assert_array_equal(O.felzenszwalb(f, dims), small[f"{name}_felz"])


def test_oracle_matches_golden_digests(O, digests):
    dims = (1024, 1024)
    m = O.add_points(O.new_mask(*dims), dims, 100, 1)
    assert digest(m) == digests["c1_mask"]
    ini = O.init_deltas(m, dims)
    for meth in ("danielsson", "fastsweep"):
        assert digest(O.propagate(meth, ini, dims, 1)) == digests[f"c1_{meth}_cw1"], meth
    bor = O.border_init(m, dims)
    assert digest(bor) == digests["c1_border"]
    assert digest(O.propagate("danielsson", bor, dims, 2)) == digests["c1_danielsson_cw2"]
    assert digest(O.felzenszwalb(O.init_distances(m, dims), dims)) == digests["c1_felz"]
    dims = (64, 64, 64)
    m = O.add_points(O.add_block(O.new_mask(*dims), dims, 6), dims, 200, 12345)
    assert digest(m) == digests["v64_mask"]
    bor = O.border_init(m, dims)
    assert digest(bor) == digests["v64_border"]
    for meth in ("danielsson", "fastsweep"):
        assert digest(O.propagate(meth, bor, dims, 2)) == digests[f"v64_{meth}_cw2"], meth


def _rand_mask(rng, dims, p, garbage=False):
    m = rng.random(tuple(reversed(dims))) < p
    words = __import__("oracle").bool_to_mask(m)
    w = dims[0]
    if garbage and w % 32:
        ws = (w + 31) // 32
        rows = words.reshape(-1, ws)
        pad = np.uint32(~np.uint32((1 << (w % 32)) - 1))
        rows[:, -1] |= rng.integers(0, 2**32, size=rows.shape[0], dtype=np.uint64).astype(np.uint32) & pad
        words = rows.reshape(-1)
    return words


@pytest.mark.parametrize("dims", [(1, 1), (1, 7), (7, 1), (31, 9), (32, 5), (33, 11), (65, 20), (100, 3)])
def test_oracle_vs_reference_2d(O, dims):
    if O.ref() is None:
        pytest.skip("reference build (oracle/_ref) not available")
    rng = np.random.default_rng(hash(dims) & 0xFFFF)
    for p in (0.0, 0.05, 0.3, 0.7, 1.0):
        for garbage in (False, True):
            m = _rand_mask(rng, dims, p, garbage)
            np.testing.assert_array_equal(O.border_init(m, dims), O.border_init(m, dims, use_ref=True))
            for inv in (False, True):
                np.testing.assert_array_equal(O.init_deltas(m, dims, inv), O.init_deltas(m, dims, inv, use_ref=True))
            ini, bor = O.init_deltas(m, dims), O.border_init(m, dims)
            for meth in ("danielsson", "fastsweep", "jumpflood", "bruteforce"):
                for cw, start in ((1, ini), (2, bor)):
                    np.testing.assert_array_equal(O.propagate(meth, start, dims, cw),
                                                  O.propagate(meth, start, dims, cw, use_ref=True),
                                                  err_msg=f"{meth} cw{cw} p{p}")
            f = O.init_distances(m, dims)
            np.testing.assert_array_equal(f, O.init_distances(m, dims, use_ref=True))
            np.testing.assert_array_equal(O.felzenszwalb(f, dims), O.felzenszwalb(f, dims, use_ref=True))


@pytest.mark.parametrize("dims", [(1, 1, 1), (5, 1, 1), (1, 4, 3), (9, 7, 5), (32, 3, 4), (33, 6, 5), (40, 1, 6)])
def test_oracle_vs_reference_3d(O, dims):
    if O.ref() is None:
        pytest.skip("reference build (oracle/_ref) not available")
    rng = np.random.default_rng(hash(dims) & 0xFFFF)
    big = np.float32(np.finfo(np.float32).max)
    for p in (0.0, 0.05, 0.3, 0.7, 1.0):
        for garbage in (False, True):
            m = _rand_mask(rng, dims, p, garbage)
            np.testing.assert_array_equal(O.border_init(m, dims), O.border_init(m, dims, use_ref=True))
            ini, bor = O.init_deltas(m, dims), O.border_init(m, dims)
            np.testing.assert_array_equal(ini, O.init_deltas(m, dims, use_ref=True))
            for meth in ("danielsson", "fastsweep", "jumpflood", "bruteforce"):
                for cw, start in ((1, ini), (2, bor)):
                    np.testing.assert_array_equal(O.propagate(meth, start, dims, cw),
                                                  O.propagate(meth, start, dims, cw, use_ref=True),
                                                  err_msg=f"{meth} cw{cw} p{p}")
            b = O.mask_to_bool(m, dims)
            f = np.where(b, np.float32(0), big).astype(np.float32)
            np.testing.assert_array_equal(O.felzenszwalb(f, dims), O.felzenszwalb(f, dims, use_ref=True))


@pytest.mark.parametrize("dims", [(31, 9), (33, 11), (65, 20), (9, 7, 5), (33, 6, 5), (40, 1, 6)])
def test_two_pass_oracle_vs_reference(O, dims):
    """The -S field's deltas (exterior and interior, cw = 1) against the reference's
    own init (both inversions) and delta methods; the float difference follows."""
    if O.ref() is None:
        pytest.skip("reference build (oracle/_ref) not available")
    rng = np.random.default_rng(sum(dims) + 17)
    for p in (0.0, 0.05, 0.3, 0.7, 1.0):
        m = _rand_mask(rng, dims, p, True)
        for meth in ("danielsson", "fastsweep", "jumpflood"):
            mine, theirs = O.sdf_two_pass(m, dims, meth), O.sdf_two_pass(m, dims, meth, use_ref=True)
            for a, b in zip(mine, theirs):
                np.testing.assert_array_equal(a, b, err_msg=f"{meth} p{p}")
            b = O.mask_to_bool(m, dims)
            dist = mine[2]
            assert (dist[b] <= 0).all() and (dist[~b] >= 0).all()


@pytest.mark.parametrize("dims", [(2, 1), (2, 6), (7, 1), (31, 9), (33, 17), (100, 3), (65, 64)])
def test_chamfer_oracle_vs_reference(O, dims):
    """Chamfer on int16 / int32 fields: tool-style inits, the int32 default that
    wraps in the reference, and arbitrary values (negative and near the maximum)."""
    if O.ref() is None:
        pytest.skip("reference build (oracle/_ref) not available")
    rng = np.random.default_rng(sum(dims) + 23)
    for p in (0.0, 0.01, 0.2, 0.9):
        m = _rand_mask(rng, dims, p, True)
        for dt, md in ((np.int16, 32767 - 16), (np.int16, 32767), (np.int32, 2**31 - 16), (np.int32, 2**31 - 1)):
            f = O.init_distances_int(m, dims, dt, md)
            np.testing.assert_array_equal(f, O.init_distances_int(m, dims, dt, md, use_ref=True))
            (a, ma), (b, mb) = O.chamfer(f, dims), O.chamfer(f, dims, use_ref=True)
            assert ma == mb == 3
            np.testing.assert_array_equal(a, b, err_msg=f"{dt} {md} p{p}")
    for dt in (np.int16, np.int32):
        info = np.iinfo(dt)
        f = rng.integers(info.min, info.max, size=tuple(reversed(dims)), dtype=np.int64, endpoint=True).astype(dt)
        np.testing.assert_array_equal(O.chamfer(f, dims)[0], O.chamfer(f, dims, use_ref=True)[0])


def test_reference_felzenszwalb_exact_range(O):
    """Where the reference's float Felzenszwalb stops being the exact EDT: rows of
    up to 4096 cells give the exact squared EDT (every intermediate an integer
    below 2^24), longer rows do not (an all-set 5000 x 3 image comes back with
    nonzero distances).  The integer EDT used to check the GPU beyond 4096 agrees
    with the reference inside that range."""
    if O.ref() is None:
        pytest.skip("reference build (oracle/_ref) not available")
    big = np.float32(np.finfo(np.float32).max)
    zero = O.felzenszwalb(np.zeros((3, 4096), np.float32), (4096, 3), use_ref=True)
    assert not zero.any()
    off = O.felzenszwalb(np.zeros((3, 5000), np.float32), (5000, 3), use_ref=True)
    assert off.any()
    rng = np.random.default_rng(4)
    for dims in ((300, 4), (100, 3, 2), (4096, 3)):
        for p in (0.0, 0.01, 0.4, 1.0):
            m = _rand_mask(rng, dims, p, False)
            b = O.mask_to_bool(m, dims)
            want = O.felzenszwalb(np.where(b, np.float32(0), big).astype(np.float32), dims, use_ref=True)
            ex = O.edt_exact_thin(m, dims)
            got = np.where(ex < 0, big, ex.astype(np.float32)).astype(np.float32)
            np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32))


def test_felzenszwalb_is_exact_edt(O):
    """The float envelope returns the exact squared EDT (so any exact EDT matches it)."""
    rng = np.random.default_rng(5)
    for dims in [(37, 29), (64, 64), (13, 9, 11), (24, 17, 20)]:
        for p in (0.001, 0.02, 0.3):
            m = _rand_mask(rng, dims, p)
            big = np.float32(np.finfo(np.float32).max)
            f = np.where(O.mask_to_bool(m, dims), np.float32(0), big).astype(np.float32)
            np.testing.assert_array_equal(O.felzenszwalb(f, dims), O.edt_brute(m, dims))


def test_generators_match_reference(O):
    if O.ref() is None:
        pytest.skip("reference build (oracle/_ref) not available")
    for dims in [(64, 64), (100, 37), (1024, 1024)]:
        np.testing.assert_array_equal(O.add_points(O.new_mask(*dims), dims, 100, 1),
                                      O.add_points(O.new_mask(*dims), dims, 100, 1, use_ref=True))
        for s in range(6):
            np.testing.assert_array_equal(O.add_block(O.new_mask(*dims), dims, s),
                                          O.add_block(O.new_mask(*dims), dims, s, use_ref=True))
    for dims in [(16, 16, 16), (40, 33, 20)]:
        np.testing.assert_array_equal(O.add_points(O.new_mask(*dims), dims, 50, 12345),
                                      O.add_points(O.new_mask(*dims), dims, 50, 12345, use_ref=True))
        for s in range(8):
            np.testing.assert_array_equal(O.add_block(O.new_mask(*dims), dims, s),
                                          O.add_block(O.new_mask(*dims), dims, s, use_ref=True))


def _readme_case(O, name):
    from PIL import Image
    img = np.asarray(Image.open(os.path.join(REF_DIR, "data", f"{name}.png")).convert("L"))
    h, w = img.shape
    mask = O.pack_bytes(img, 128, True)          # the tool's defaults (Tool.cpp:1774-1775)
    bor = O.border_init(mask, (w, h))
    dl = O.propagate("danielsson", bor, (w, h), 2)
    dist = O.deltas_to_dist(dl, (w, h), 2, sign_mask=mask)
    max_len = 0.25 * max(w, h) * 2                # Tool.cpp:1973-1974, signed border: maxLen * 2
    v = np.clip(dist * 2 / np.float32(max_len), -1, 1)   # deltas_to_dist halves cw=2 lengths
    enc = np.rint(128 + v.astype(np.float32) * 127).astype(np.int32)
    want = np.asarray(Image.open(os.path.join(REF_DIR, "images", f"{name}-sdf.png")).convert("L")).astype(np.int32)
    return enc, want


@pytest.mark.parametrize("name", ["tiger", "kiwi"])
def test_readme_sdf_images_within_one_level(O, name):
    if REF_DIR is None:
        pytest.skip("reference checkout not present (set DOL_REFERENCE_DIR)")
    enc, want = _readme_case(O, name)
    diff = np.abs(enc - want)
    assert diff.max() <= 1, f"max grey-level difference {diff.max()}"


# ---- occlusion sweeps ----------------------------------------------------------------------

@pytest.mark.parametrize("dims", [(1, 1), (1, 7), (7, 1), (31, 9), (33, 20), (64, 64), (100, 37),
                                  (1, 1, 1), (5, 1, 3), (9, 7, 5), (33, 6, 5), (24, 20, 16)])
def test_occlusion_matches_reference(O, dims):
    if O.ref() is None:
        pytest.skip("reference build (oracle/_ref) absent")
    rng = np.random.default_rng(sum(dims) + 41)
    for p in (0.0, 0.05, 0.3, 0.8, 1.0):
        m = O.bool_to_mask(rng.random(tuple(reversed(dims))) < p)
        dw = O.init_dirw(m, dims)
        np.testing.assert_array_equal(dw, O.init_dirw(m, dims, use_ref=True))
        got = O.occlusion_sweep(dw, dims)
        want = O.occlusion_sweep(dw, dims, use_ref=True)
        np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32), err_msg=f"{dims} p={p}")
        if len(dims) == 3:
            prior = rng.random(dw.shape).astype(np.float32)   # cells the reference leaves unwritten keep this
            got = O.occlusion_sweep_io(dw, prior, dims)
            want = O.occlusion_sweep_io(dw, prior, dims, use_ref=True)
            np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32), err_msg=f"io {dims} p={p}")


# ---- mesh voxeliser -------------------------------------------------------------------------

def _tri_file():
    return os.path.join(os.path.dirname(HERE), "oracle", "_ref", "plant2.tri")


@pytest.mark.parametrize("dims", [(32, 32, 32), (64, 64, 64), (100, 80, 60), (33, 17, 70)])
def test_voxelize_matches_reference(O, dims):
    if O.ref() is None:
        pytest.skip("reference build (oracle/_ref) absent")
    rng = np.random.default_rng(sum(dims))
    cases = [O.random_triangles(rng, 400), O.random_triangles(rng, 50, scale=(0.3, 1.5))]
    if os.path.exists(_tri_file()):
        cases.append(O.load_tri(_tri_file()))
    for idx, v, bb in cases:
        got = O.voxelize(idx, v, bb, dims)
        want = O.voxelize(idx, v, bb, dims, use_ref=True)
        np.testing.assert_array_equal(got, want)
        assert want.any()
        # ORs into what the mask already holds
        prior = O.bool_to_mask(rng.random(tuple(reversed(dims))) < 0.01)
        np.testing.assert_array_equal(O.voxelize(idx, v, bb, dims, mask=prior),
                                      O.voxelize(idx, v, bb, dims, mask=prior, use_ref=True))
