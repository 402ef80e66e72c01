"""ctypes binding for the CPU oracle (TEST INFRASTRUCTURE ONLY).

Loads ``oracle/liboracle.so`` (the C restatement in ``dol_oracle.c``) and,
when present, ``oracle/_ref/libdolref.so`` (the unmodified reference library
compiled by ``oracle/Makefile``).  Only tests/, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of bench.py import this module; the CUDA library never
does.

Arrays are numpy: masks ``uint32[words]``, 2D deltas ``int16[h, w, 2]``, 3D
deltas ``int16[d, h, w, 3]``, distances ``float32``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
MAX2 = 32767
MAX3 = 25000

_lib = None
_ref = None


def build() -> None:
    """Compile liboracle.so (and _ref/libdolref.so when the reference sources exist)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        _lib = C.CDLL(path)
    return _lib


def ref():
    """The reference library build, or None when oracle/_ref was not built."""
    global _ref
    if _ref is None:
        path = os.path.join(HERE, "_ref", "libdolref.so")
        if not os.path.exists(path):
            return None
        _ref = C.CDLL(path)
    return _ref


def mask_words(w, h, d=1):
    return ((w + 31) // 32) * h * d


def new_mask(w, h, d=1):
    return np.zeros(mask_words(w, h, d), dtype=np.uint32)


def _i(*xs):
    return [C.c_int(int(x)) for x in xs]


# ---- generators ---------------------------------------------------------------

def add_points(mask, dims, n, seed, use_ref=False):
    L = ref() if use_ref else lib()
    pre = "ref_" if use_ref else "dolo_"
    if len(dims) == 2:
        getattr(L, pre + "add_points_2d")(*_i(*dims, n), C.c_uint32(seed), _p(mask))
    else:
        getattr(L, pre + "add_points_3d")(*_i(*dims, n), C.c_uint32(seed), _p(mask))
    return mask


def add_block(mask, dims, sides, use_ref=False):
    L = ref() if use_ref else lib()
    pre = "ref_" if use_ref else "dolo_"
    fn = getattr(L, pre + ("add_block_2d" if len(dims) == 2 else "add_block_3d"))
    fn(*_i(*dims, sides), _p(mask))
    return mask


def pack_bytes(img, threshold=128, less_than=True):
    h, w = img.shape
    img = np.ascontiguousarray(img, dtype=np.uint8)
    m = new_mask(w, h)
    lib().dolo_pack_bytes(*_i(w, h), _p(img), *_i(threshold, 1 if less_than else 0), _p(m))
    return m


# ---- delta methods --------------------------------------------------------------

def _deltas(dims):
    if len(dims) == 2:
        w, h = dims
        return np.empty((h, w, 2), dtype=np.int16)
    w, h, d = dims
    return np.empty((d, h, w, 3), dtype=np.int16)


def init_deltas(mask, dims, invert=False, use_ref=False):
    out = _deltas(dims)
    nd = len(dims)
    if use_ref:
        getattr(ref(), f"ref_init_deltas_{nd}d")(*_i(*dims), _p(mask), _p(out), C.c_int(int(invert)))
    else:
        getattr(lib(), f"dolo_init_deltas_{nd}d")(*_i(*dims), _p(mask), _p(out), C.c_int(int(invert)))
    return out


def border_init(mask, dims, use_ref=False):
    out = _deltas(dims)
    nd = len(dims)
    name = ("ref_" if use_ref else "dolo_") + f"border_init_{nd}d"
    getattr(ref() if use_ref else lib(), name)(*_i(*dims), _p(mask), _p(out))
    return out


def propagate(method, deltas, dims, cw, use_ref=False, exact_bf3=False):
    """Run a delta method in place on a copy; returns the new array."""
    out = np.ascontiguousarray(deltas).copy()
    nd = len(dims)
    if use_ref:
        fn = getattr(ref(), f"ref_{method}_{nd}d")
        fn(*_i(*dims), _p(out), C.c_int(cw))
        return out
    L = lib()
    if method == "jumpflood":
        tmp = np.empty_like(out)
        getattr(L, f"dolo_jumpflood_{nd}d")(*_i(*dims), _p(out), C.c_int(cw), _p(tmp))
    elif method == "bruteforce" and nd == 3:
        L.dolo_bruteforce_3d(*_i(*dims), _p(out), C.c_int(cw), C.c_int(1 if exact_bf3 else 0))
    else:
        getattr(L, f"dolo_{method}_{nd}d")(*_i(*dims), _p(out), C.c_int(cw))
    return out


def deltas_to_dist(deltas, dims, cw, sign_mask=None):
    nd = len(dims)
    out = np.empty(deltas.shape[:-1], dtype=np.float32)
    sm = _p(sign_mask) if sign_mask is not None else None
    getattr(lib(), f"dolo_deltas_to_dist_{nd}d")(*_i(*dims), _p(np.ascontiguousarray(deltas)),
                                                 C.c_int(cw), sm, _p(out))
    return out


def sdf_two_pass(mask, dims, method, use_ref=False):
    """The tool's -S field (GenerateSignedDistance, DistanceOcclusionTool.cpp:1082-1123
    2D, :1197-1232 3D): deltas to set cells (InitDeltasFromBitMask, invert=false) and to
    clear cells (invert=true), each through FindDeltas(method) with cw = 1 (:711-739),
    then Dist(d0) - Dist(d1) in float (:54-61, :1136).  Returns (d0, d1, dist)."""
    d0 = propagate(method, init_deltas(mask, dims, False, use_ref=use_ref), dims, 1, use_ref=use_ref)
    d1 = propagate(method, init_deltas(mask, dims, True, use_ref=use_ref), dims, 1, use_ref=use_ref)
    dist = (deltas_to_dist(d0, dims, 1) - deltas_to_dist(d1, dims, 1)).astype(np.float32)
    return d0, d1, dist


# ---- accuracy against BruteForce ----------------------------------------------------------

ERR_EDGES = np.array([0.0, 1e-6, 0.05, 0.1, 0.2, 0.3, 0.4, 0.5, 0.75, 1.0, np.inf], dtype=np.float64)


def error_histogram(deltas, refs, dims, edges=ERR_EDGES):
    """The tool's error measure (PrintError, DistanceOcclusionTool.cpp:265-287): per cell
    |Dist(delta) - Dist(ref)| in float, Dist = sqrtf of the int32 squared length (:46-61).
    Returns (counts per [edges[i], edges[i+1]), max error)."""
    a = deltas_to_dist(np.ascontiguousarray(deltas), dims, 1)
    b = deltas_to_dist(np.ascontiguousarray(refs), dims, 1)
    err = np.abs(a - b).astype(np.float32)
    counts, _ = np.histogram(err.astype(np.float64), bins=edges)
    return counts, float(err.max()) if err.size else 0.0


# ---- Chamfer (integer distances) ----------------------------------------------------------

def init_distances_int(mask, dims, dtype, max_d, use_ref=False):
    """InitDistancesFromBitMask, int16 / int32 overloads (DistanceOcclusionLib.cpp:183-222)."""
    w, h = dims
    dt = np.dtype(dtype)
    out = np.empty((h, w), dtype=dt)
    tag = "i16" if dt == np.int16 else "i32"
    cval = C.c_int16(int(max_d)) if dt == np.int16 else C.c_int32(int(max_d))
    getattr(ref() if use_ref else lib(), ("ref_" if use_ref else "dolo_") + f"init_distances_2d_{tag}")(
        *_i(w, h), _p(mask), _p(out), cval)
    return out


def chamfer(dist, dims, use_ref=False):
    """Chamfer 3-4 on a copy of an int16 / int32 field (DistanceOcclusionLib.cpp:916-1016);
    returns (field, multiplier)."""
    w, h = dims
    out = np.ascontiguousarray(dist).copy()
    tag = "i16" if out.dtype == np.int16 else "i32"
    m = getattr(ref() if use_ref else lib(), ("ref_" if use_ref else "dolo_") + f"chamfer_2d_{tag}")(
        *_i(w, h), _p(out))
    return out, m


# ---- Felzenszwalb ---------------------------------------------------------------------

def init_distances(mask, dims, use_ref=False):
    w, h = dims
    out = np.empty((h, w), dtype=np.float32)
    if use_ref:
        ref().ref_init_distances_2d(*_i(w, h), _p(mask), _p(out))
    else:
        lib().dolo_init_distances_2d(*_i(w, h), _p(mask), _p(out), C.c_float(np.finfo(np.float32).max))
    return out


def felzenszwalb(dist, dims, use_ref=False, threads=1):
    """Squared EDT of a float field (0 at seeds, FLT_MAX elsewhere), in place on a copy."""
    out = np.ascontiguousarray(dist, dtype=np.float32).copy()
    n = max(dims)
    if use_ref:
        if len(dims) == 2:
            ref().ref_felzenszwalb_2d(*_i(*dims), _p(out))
        else:
            ref().ref_felzenszwalb_3d(*_i(*dims), _p(out), C.c_int(threads))
        return out
    v = np.empty(n, dtype=np.int32)
    z = np.empty(n + 1, dtype=np.float32)
    if len(dims) == 2:
        td = np.empty(out.size, dtype=np.float32)
        lib().dolo_felzenszwalb_2d(*_i(*dims), _p(out), _p(td), _p(v), _p(z))
    else:
        td = np.empty(n, dtype=np.float32)
        lib().dolo_felzenszwalb_3d(*_i(*dims), _p(out), _p(td), _p(v), _p(z))
    return out


def mask_to_bool(mask, dims):
    """Unpack a padded bitmask to bool[h, w] / bool[d, h, w]."""
    w = dims[0]
    ws = (w + 31) // 32
    rows = mask.reshape(-1, ws)
    bits = np.unpackbits(rows.view(np.uint8).reshape(rows.shape[0], ws * 4), axis=1, bitorder="little")
    b = bits[:, :w].astype(bool)
    return b.reshape(tuple(reversed(dims)))


def bool_to_mask(b):
    """Pack bool[h, w] / bool[d, h, w] (x fastest) into a padded bitmask."""
    b = np.asarray(b, dtype=bool)
    w = b.shape[-1]
    ws = (w + 31) // 32
    rows = b.reshape(-1, w)
    pad = np.zeros((rows.shape[0], ws * 32), dtype=np.uint8)
    pad[:, :w] = rows
    packed = np.packbits(pad, axis=1, bitorder="little")
    return np.ascontiguousarray(packed).view(np.uint32).reshape(-1).copy()


def sdf_signed_felzenszwalb(mask, dims):
    """Two-pass signed Felzenszwalb (distance to occupied minus distance to empty),
    the orthodox -S convention of DistanceOcclusionTool.cpp:1036, built from the
    restated EDT: positive outside, negative inside."""
    b = mask_to_bool(mask, dims)
    big = np.float32(np.finfo(np.float32).max)
    f_occ = np.where(b, np.float32(0), big).astype(np.float32)
    f_emp = np.where(b, big, np.float32(0)).astype(np.float32)
    e_occ = felzenszwalb(f_occ, dims)
    e_emp = felzenszwalb(f_emp, dims)
    return (np.sqrt(e_occ) - np.sqrt(e_emp)).astype(np.float32)


def edt_exact_thin(mask, dims):
    """Exact squared EDT in int64 for fields with few rows per line set (h * d
    small): exact distance along x to the nearest set cell of each row, then the
    min over all rows of dx^2 + dy^2 + dz^2.  Used where a row is longer than the
    reference's float envelope keeps exact (about 4096 cells: its q*q passes 2^24
    and the intersections round), i.e. as the exact EDT rather than the
    reference's.  Returns int64 with -1 where no set cell exists."""
    b = mask_to_bool(mask, dims)
    shp = b.shape
    w = dims[0]
    rows = b.reshape(-1, w)
    inf = np.int64(1) << 60
    xs = np.arange(w)
    dx = np.full(rows.shape, inf, np.int64)
    for r in range(rows.shape[0]):
        idx = np.nonzero(rows[r])[0]
        if idx.size:
            pos = np.searchsorted(idx, xs)
            left = np.where(pos > 0, xs - idx[np.maximum(pos - 1, 0)], inf)
            right = np.where(pos < idx.size, idx[np.minimum(pos, idx.size - 1)] - xs, inf)
            dx[r] = np.minimum(left, right)
    h = dims[1]
    d = dims[2] if len(dims) == 3 else 1
    out = np.full(rows.shape, inf, np.int64)
    for r in range(rows.shape[0]):
        z, y = divmod(r, h)
        for r2 in range(rows.shape[0]):
            z2, y2 = divmod(r2, h)
            cand = np.where(dx[r2] < inf, dx[r2] ** 2 + (y - y2) ** 2 + (z - z2) ** 2, inf)
            out[r] = np.minimum(out[r], cand)
    out = np.where(out >= inf, -1, out)
    return out.reshape(shp)


def sdf_signed_exact_thin(mask, dims):
    """Signed field (distance to set cells minus distance to clear cells) from the
    exact EDT of edt_exact_thin, in float32 as the GPU forms it."""
    b = mask_to_bool(mask, dims)
    inv = bool_to_mask(~b) if b.ndim == 2 else bool_to_mask(~b)
    big = np.float32(np.finfo(np.float32).max)
    def f(e):
        return np.where(e < 0, big, e.astype(np.float32)).astype(np.float32)
    e_occ, e_emp = f(edt_exact_thin(mask, dims)), f(edt_exact_thin(inv, dims))
    return (np.sqrt(e_occ) - np.sqrt(e_emp)).astype(np.float32)


def edt_brute(mask, dims):
    d3 = list(dims) + [1] * (3 - len(dims))
    out = np.empty(d3[0] * d3[1] * d3[2], dtype=np.float32)
    lib().dolo_edt_brute(*_i(*d3), _p(mask), _p(out))
    return out.reshape(tuple(reversed(dims)))


# ---- occlusion ---------------------------------------------------------------------------

def init_dirw(mask, dims, use_ref=False):
    """InitDirWFromBitMask: float32[planes, (d,) h, w], planes = 4 (2D) / 8 (3D)."""
    planes = 4 if len(dims) == 2 else 8
    out = np.empty((planes,) + tuple(reversed(dims)), dtype=np.float32)
    if use_ref:
        if len(dims) == 2:
            ref().ref_init_dirw_2d(*_i(*dims), _p(mask), _p(out))
        else:
            ref().ref_init_dirw_3d(*_i(*dims), _p(mask), _p(out))
    else:
        d3 = list(dims) + [1] * (3 - len(dims))
        lib().dolo_init_dirw(*_i(*d3), C.c_int(planes), _p(mask), _p(out))
    return out


def occlusion_sweep(dirw, dims, use_ref=False):
    """OcclusionSweep in place (2D quadrants / 3D octants), on a copy."""
    out = np.ascontiguousarray(dirw, dtype=np.float32).copy()
    pre, L = ("ref_", ref()) if use_ref else ("dolo_", lib())
    if len(dims) == 2:
        getattr(L, pre + "occlusion_sweep_2d")(*_i(*dims), _p(out))
    else:
        getattr(L, pre + "occlusion_sweep_3d")(*_i(*dims), _p(out))
    return out


def occlusion_sweep_io(dirw_in, dirw_out, dims, use_ref=False):
    """OcclusionSweep(w, h, d, in, out): octant occlusion of `in` written to a copy of `out`."""
    src = np.ascontiguousarray(dirw_in, dtype=np.float32)
    out = np.ascontiguousarray(dirw_out, dtype=np.float32).copy()
    pre, L = ("ref_", ref()) if use_ref else ("dolo_", lib())
    getattr(L, pre + "occlusion_sweep_3d_io")(*_i(*dims), _p(src), _p(out))
    return out


# ---- mesh voxeliser ------------------------------------------------------------------------

def load_tri(path):
    """A triangle file written by oracle/_ref/mesh_dump: (indices int32[t, 3],
    vertices float32[v, 3], bbox float32[6])."""
    raw = np.fromfile(path, dtype=np.uint8)
    nt, nv = np.frombuffer(raw[:8].tobytes(), np.int32)
    bbox = np.frombuffer(raw[8:32].tobytes(), np.float32).copy()
    o = 32
    verts = np.frombuffer(raw[o:o + 12 * nv].tobytes(), np.float32).reshape(nv, 3).copy()
    o += 12 * nv
    idx = np.frombuffer(raw[o:o + 12 * nt].tobytes(), np.int32).reshape(nt, 3).copy()
    return idx, verts, bbox


def voxelize(indices, vertices, bbox, dims, mask=None, use_ref=False):
    """CreateBitMaskFromTriangles: ORs the touched cells into `mask` (a fresh
    zero mask by default); returns the mask."""
    w, h, d = dims
    m = new_mask(w, h, d) if mask is None else mask.copy()
    idx = np.ascontiguousarray(indices, np.int32)
    v = np.ascontiguousarray(vertices, np.float32)
    bb = np.ascontiguousarray(bbox, np.float32)
    if use_ref:
        ref().ref_voxelize(C.c_int(idx.shape[0]), _p(idx), _p(v), _p(bb), *_i(w, h, d), _p(m))
    else:
        lib().dolo_voxelize(C.c_int(idx.shape[0]), _p(idx), _p(v), _p(bb), *_i(w, h, d), _p(m))
    return m


def random_triangles(rng, n, scale=(0.002, 0.3), nverts=None):
    """A soup of n triangles in the unit cube: sizes log-uniform in `scale`,
    some degenerate (repeated or collinear vertices); returns (indices,
    vertices, bbox) with bbox the vertices' bounds."""
    c = rng.random((n, 1, 3))
    size = np.exp(rng.uniform(np.log(scale[0]), np.log(scale[1]), (n, 1, 1)))
    tri = c + (rng.random((n, 3, 3)) - 0.5) * size
    k = max(1, n // 40)
    tri[:k, 2] = tri[:k, 1]                                        # repeated vertex
    tri[k:2 * k, 2] = 2 * tri[k:2 * k, 1] - tri[k:2 * k, 0]          # collinear
    verts = tri.reshape(-1, 3).astype(np.float32)
    idx = np.arange(3 * n, dtype=np.int32).reshape(n, 3)
    perm = rng.permutation(3 * n).astype(np.int32)                # shuffled vertex order, indexed
    vs = np.empty_like(verts)
    vs[perm] = verts
    idx = perm[idx]
    bbox = np.concatenate([verts.min(0), verts.max(0)]).astype(np.float32)
    return idx, vs, bbox
