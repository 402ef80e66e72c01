"""dol_b200 -- Python host side of the B200 distance-field library.

A thin ctypes layer over ``libdol_b200.so`` (the C ABI in include/dol_b200.h)
that mirrors the reference's DOL interface (DistanceOcclusionLib.h) on torch
CUDA tensors: torch provides device memory and streams, every computation runs
in the library's CUDA kernels.  There is no CPU fallback: if the library
cannot be loaded, every call raises.

Layouts follow the reference: masks are uint32 words with rows padded to
(w+31)//32 words (torch.int32 tensors holding the same bits); 2D deltas are
int16 tensors of shape (h, w, 2), 3D deltas (d, h, w, 3); distances float32.

The directory name contains a hyphen, so import it by path::

    import importlib.util, sys
    spec = importlib.util.spec_from_file_location(
        "dol_b200", "<repo>/distance-occlusion_b200/__init__.py")
    dol = importlib.util.module_from_spec(spec); sys.modules["dol_b200"] = dol
    spec.loader.exec_module(dol)
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import os

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG_DIR, "libdol_b200.so")

# status codes (dol_status)
OK, ERR_INVALID_ARG, ERR_CUDA, ERR_NO_MEMORY, ERR_TIMEOUT, ERR_UNSUPPORTED = range(6)
# methods (dol_method), numbered as the reference tool's -m
DANIELSSON, FASTSWEEP, JUMPFLOOD, FELZENSZWALB = 0, 1, 2, 5
METHODS = {"danielsson": DANIELSSON, "fastsweep": FASTSWEEP, "jumpflood": JUMPFLOOD, "felzenszwalb": FELZENSZWALB}
# EDT output forms
EDT_SQUARED, EDT_DIST, EDT_SIGNED = 0, 1, 2
MAX_DELTA2 = 32767
MAX_DELTA3 = 25000


class DolError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"dol_b200 error {status}: {message}")
        self.status = status


_lib = None


def build(force: bool = False) -> str:
    """Compile the CUDA library in-tree (nvcc, sm_100a)."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("_dol_build", os.path.join(PKG_DIR, "build.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.build(force=force)


def lib():
    """The loaded CUDA library; raises if it is missing."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise DolError(ERR_UNSUPPORTED, f"CUDA library not built: {LIB_PATH} (run distance-occlusion_b200/build.py)")
        L = C.CDLL(LIB_PATH)
        L.dol_last_error.restype = C.c_char_p
        L.dol_status_string.restype = C.c_char_p
        for name in ("dol_mask_words", "dol_jumpflood_2d_workspace_size", "dol_jumpflood_3d_workspace_size",
                     "dol_fastsweep_3d_workspace_size", "dol_felzenszwalb_2d_workspace_size",
                     "dol_edt_mask_2d_workspace_size", "dol_edt_mask_3d_workspace_size", "dol_sdf_workspace_size",
                     "dol_sdf_two_pass_workspace_size",
                     "dol_batch_workspace_size", "dol_sites_backward_workspace_size",
                     "dol_danielsson_workspace_size"):
            getattr(L, name).restype = C.c_size_t
        _lib = L
    return _lib


def check(status: int) -> None:
    if status != OK:
        raise DolError(status, lib().dol_last_error().decode(errors="replace"))


def sync(stream=None) -> None:
    """Wait for `stream` (default: torch's current stream) and report device-side errors."""
    check(lib().dol_sync(_stream(stream)))


# ---- helpers ----------------------------------------------------------------------------------

def _torch():
    import torch
    return torch


def _stream(stream=None):
    if stream is None:
        torch = _torch()
        if not torch.cuda.is_available():
            return None
        stream = torch.cuda.current_stream()
    return C.c_void_p(stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream))


def _ptr(t):
    if t is None:
        return None
    if not t.is_cuda:
        raise DolError(ERR_INVALID_ARG, "tensor is not on a CUDA device")
    if not t.is_contiguous():
        raise DolError(ERR_INVALID_ARG, "tensor must be contiguous")
    return C.c_void_p(t.data_ptr())


def _ints(*xs):
    return [C.c_int(int(x)) for x in xs]


def mask_words(w, h, d=1):
    return ((w + 31) // 32) * h * d


def _dims(dims):
    dims = tuple(int(x) for x in dims)
    if len(dims) not in (2, 3):
        raise DolError(ERR_INVALID_ARG, "dims must be (w, h) or (w, h, d)")
    return dims


def empty_deltas(dims, device="cuda"):
    torch = _torch()
    dims = _dims(dims)
    if len(dims) == 2:
        return torch.empty((dims[1], dims[0], 2), dtype=torch.int16, device=device)
    return torch.empty((dims[2], dims[1], dims[0], 3), dtype=torch.int16, device=device)


def empty_field(dims, device="cuda"):
    torch = _torch()
    return torch.empty(tuple(reversed(_dims(dims))), dtype=torch.float32, device=device)


# ---- reference-shaped API (DOL::*) -------------------------------------------------------------

def add_points(mask_host, dims, n, seed):
    """BitMaskAddPoints on a host numpy uint32 mask (the reference's LCG)."""
    dims = _dims(dims)
    p = mask_host.ctypes.data_as(C.c_void_p)
    if len(dims) == 2:
        lib().dol_add_points_2d(*_ints(*dims, n), C.c_uint32(seed), p)
    else:
        lib().dol_add_points_3d(*_ints(*dims, n), C.c_uint32(seed), p)
    return mask_host


def add_block(mask_host, dims, sides):
    """BitMaskAddBlock on a host numpy uint32 mask."""
    dims = _dims(dims)
    p = mask_host.ctypes.data_as(C.c_void_p)
    fn = lib().dol_add_block_2d if len(dims) == 2 else lib().dol_add_block_3d
    fn(*_ints(*dims, sides), p)
    return mask_host


def pack_bytemask(img, threshold=128, less_than=True, stream=None):
    """Byte image (h, w) or volume (d, h, w) uint8 CUDA tensor -> bitmask (BitMaskFromImageFile)."""
    torch = _torch()
    shape = tuple(img.shape)
    w = shape[-1]
    h = shape[-2]
    d = shape[0] if len(shape) == 3 else 1
    out = torch.empty(mask_words(w, h, d), dtype=torch.int32, device=img.device)
    check(lib().dol_pack_bytemask(*_ints(w, h, d), _ptr(img), *_ints(threshold, 1 if less_than else 0),
                                  _ptr(out), _stream(stream)))
    return out


def init_distances(mask, dims, max_d=None, stream=None):
    """InitDistancesFromBitMask (float): 0 on set cells, max_d (FLT_MAX) elsewhere."""
    import numpy as np
    dims = _dims(dims)
    out = empty_field(dims, mask.device)
    md = float(np.finfo(np.float32).max) if max_d is None else float(max_d)
    check(lib().dol_init_distances_2d(*_ints(*dims), _ptr(mask), _ptr(out), C.c_float(md), _stream(stream)))
    return out


def init_distances_int(mask, dims, dtype="int16", max_d=None, out=None, stream=None):
    """InitDistancesFromBitMask, int16 / int32 overloads: 0 on set bits, max_d elsewhere
    (default INT16_MAX - 16 / INT32_MAX - 16, the margin the tool keeps for Chamfer's adds)."""
    torch = _torch()
    w, h = _dims(dims)
    td = torch.int16 if str(dtype).endswith("int16") else torch.int32
    if max_d is None:
        max_d = 32767 - 16 if td == torch.int16 else 2**31 - 1 - 16
    if out is None:
        out = torch.empty((h, w), dtype=td, device=mask.device)
    if td == torch.int16:
        check(lib().dol_init_distances_2d_i16(*_ints(w, h), _ptr(mask), _ptr(out), C.c_int16(int(max_d)), _stream(stream)))
    else:
        check(lib().dol_init_distances_2d_i32(*_ints(w, h), _ptr(mask), _ptr(out), C.c_int32(int(max_d)), _stream(stream)))
    return out


def chamfer(dist, dims, stream=None):
    """Chamfer 3-4 in place on an int16 / int32 field; returns the multiplier (3)."""
    torch = _torch()
    w, h = _dims(dims)
    m = C.c_int(0)
    fn = lib().dol_chamfer_2d_i16 if dist.dtype == torch.int16 else lib().dol_chamfer_2d_i32
    check(fn(*_ints(w, h), _ptr(dist), C.byref(m), _stream(stream)))
    return m.value


def init_deltas(mask, dims, invert=False, out=None, stream=None):
    """InitDeltasFromBitMask."""
    dims = _dims(dims)
    out = empty_deltas(dims, mask.device) if out is None else out
    fn = lib().dol_init_deltas_2d if len(dims) == 2 else lib().dol_init_deltas_3d
    check(fn(*_ints(*dims), _ptr(mask), _ptr(out), C.c_int(1 if invert else 0), _stream(stream)))
    return out


def init_border(mask, dims, out=None, stream=None):
    """InitBorderDeltasFromBitMask (signed, half-cell deltas)."""
    dims = _dims(dims)
    out = empty_deltas(dims, mask.device) if out is None else out
    fn = lib().dol_init_border_2d if len(dims) == 2 else lib().dol_init_border_3d
    check(fn(*_ints(*dims), _ptr(mask), _ptr(out), _stream(stream)))
    return out


def danielsson(deltas, dims, cw=1, stream=None):
    dims = _dims(dims)
    fn = lib().dol_danielsson_2d if len(dims) == 2 else lib().dol_danielsson_3d
    check(fn(*_ints(*dims), _ptr(deltas), C.c_int(cw), _stream(stream)))
    return deltas


def fastsweep(deltas, dims, cw=1, workspace=None, stream=None):
    dims = _dims(dims)
    if len(dims) == 2:
        check(lib().dol_fastsweep_2d(*_ints(*dims), _ptr(deltas), C.c_int(cw), _stream(stream)))
    else:
        wsb = workspace.numel() * workspace.element_size() if workspace is not None else 0
        check(lib().dol_fastsweep_3d(*_ints(*dims), _ptr(deltas), C.c_int(cw), _ptr(workspace),
                                     C.c_size_t(wsb), _stream(stream)))
    return deltas


def jumpflood(deltas, dims, cw=1, workspace=None, stream=None):
    dims = _dims(dims)
    wsb = workspace.numel() * workspace.element_size() if workspace is not None else 0
    fn = lib().dol_jumpflood_2d if len(dims) == 2 else lib().dol_jumpflood_3d
    check(fn(*_ints(*dims), _ptr(deltas), C.c_int(cw), _ptr(workspace), C.c_size_t(wsb), _stream(stream)))
    return deltas


def propagate(method, deltas, dims, cw=1, stream=None):
    """FindDeltas dispatch (DistanceOcclusionTool.cpp:711-739 / :937-965)."""
    m = METHODS.get(method, method)
    if m == DANIELSSON:
        return danielsson(deltas, dims, cw, stream=stream)
    if m == FASTSWEEP:
        return fastsweep(deltas, dims, cw, stream=stream)
    if m == JUMPFLOOD:
        return jumpflood(deltas, dims, cw, stream=stream)
    raise DolError(ERR_INVALID_ARG, f"not a delta method: {method}")


def felzenszwalb(dist, dims, stream=None):
    """DOL::Felzenszwalb(w, h, float[]): in-place squared distance transform of any float field."""
    dims = _dims(dims)
    if len(dims) != 2:
        raise DolError(ERR_UNSUPPORTED, "the general float transform is 2D, as in the reference")
    check(lib().dol_felzenszwalb_2d(*_ints(*dims), _ptr(dist), None, C.c_size_t(0), _stream(stream)))
    return dist


def edt_mask(mask, dims, form=EDT_DIST, out=None, workspace=None, stream=None):
    """Exact EDT from a bitmask (Felzenszwalb path): EDT_SQUARED / EDT_DIST / EDT_SIGNED."""
    dims = _dims(dims)
    out = empty_field(dims, mask.device) if out is None else out
    wsb = workspace.numel() * workspace.element_size() if workspace is not None else 0
    if len(dims) == 2:
        check(lib().dol_edt_mask_2d(*_ints(*dims), _ptr(mask), _ptr(out), C.c_int(form), _ptr(workspace),
                                    C.c_size_t(wsb), _stream(stream)))
    else:
        check(lib().dol_edt_mask_3d(*_ints(*dims), _ptr(mask), _ptr(out), C.c_int(form), _ptr(workspace),
                                    C.c_size_t(wsb), _stream(stream)))
    return out


def edt_mask_host(mask_np, dims, form=EDT_DIST):
    """Mask-driven 3D EDT with host buffers (dol_edt_mask_3d_host): numpy mask in,
    numpy float32 field out; the copy back overlaps the last pass."""
    w, h, d = _dims(dims)
    m = np.ascontiguousarray(mask_np, dtype=np.uint32)
    out = np.empty((d, h, w), dtype=np.float32)
    check(lib().dol_edt_mask_3d_host(*_ints(w, h, d), C.c_void_p(m.ctypes.data), C.c_void_p(out.ctypes.data),
                                     C.c_int(form)))
    return out


def deltas_to_dist(deltas, dims, cw=1, sign_mask=None, out=None, stream=None):
    dims = _dims(dims)
    out = empty_field(dims, deltas.device) if out is None else out
    fn = lib().dol_deltas_to_dist_2d if len(dims) == 2 else lib().dol_deltas_to_dist_3d
    check(fn(*_ints(*dims), _ptr(deltas), C.c_int(cw), _ptr(sign_mask), _ptr(out), _stream(stream)))
    return out


def sdf(mask, dims, method="danielsson", want_deltas=True, want_dist=True, workspace=None, stream=None):
    """Signed border-initialised field in one call (GenerateSignedDistanceBorder)."""
    dims = _dims(dims)
    m = METHODS.get(method, method)
    dl = empty_deltas(dims, mask.device) if (want_deltas and m != FELZENSZWALB) else None
    df = empty_field(dims, mask.device) if want_dist else None
    wsb = workspace.numel() * workspace.element_size() if workspace is not None else 0
    if len(dims) == 2:
        check(lib().dol_sdf_2d(*_ints(*dims), _ptr(mask), C.c_int(m), _ptr(dl), _ptr(df), _ptr(workspace),
                               C.c_size_t(wsb), _stream(stream)))
    else:
        check(lib().dol_sdf_3d(*_ints(*dims), _ptr(mask), C.c_int(m), _ptr(dl), _ptr(df), _ptr(workspace),
                               C.c_size_t(wsb), _stream(stream)))
    return dl, df


def sdf_two_pass(mask, dims, method="danielsson", want_deltas=True, want_dist=True, workspace=None, stream=None):
    """Two-pass signed field (the tool's -S path, GenerateSignedDistance):
    exterior deltas (to set cells), interior deltas (to clear cells), both with
    cw = 1, and Dist(exterior) - Dist(interior).  Returns (exterior, interior,
    dist); the deltas are None unless want_deltas."""
    dims = _dims(dims)
    m = METHODS.get(method, method)
    de = empty_deltas(dims, mask.device) if want_deltas else None
    di = empty_deltas(dims, mask.device) if want_deltas else None
    df = empty_field(dims, mask.device) if want_dist else None
    wsb = workspace.numel() * workspace.element_size() if workspace is not None else 0
    if len(dims) == 2:
        check(lib().dol_sdf_two_pass_2d(*_ints(*dims), _ptr(mask), C.c_int(m), _ptr(de), _ptr(di), _ptr(df),
                                        _ptr(workspace), C.c_size_t(wsb), _stream(stream)))
    else:
        check(lib().dol_sdf_two_pass_3d(*_ints(*dims), _ptr(mask), C.c_int(m), _ptr(de), _ptr(di), _ptr(df),
                                        _ptr(workspace), C.c_size_t(wsb), _stream(stream)))
    return de, di, df


def sdf_host(mask_np, dims, method="danielsson", want_deltas=True, want_dist=True):
    """Host buffers in and out (dol_sdf_*_host): numpy in, numpy out."""
    import numpy as np
    dims = _dims(dims)
    m = METHODS.get(method, method)
    mask_np = np.ascontiguousarray(mask_np, dtype=np.uint32)
    cells = int(np.prod(dims))
    dl = None
    if want_deltas and m != FELZENSZWALB:
        dl = np.empty(tuple(reversed(dims)) + (len(dims),), dtype=np.int16)
    df = np.empty(tuple(reversed(dims)), dtype=np.float32) if want_dist else None
    pd = dl.ctypes.data_as(C.c_void_p) if dl is not None else None
    pf = df.ctypes.data_as(C.c_void_p) if df is not None else None
    pm = mask_np.ctypes.data_as(C.c_void_p)
    if len(dims) == 2:
        check(lib().dol_sdf_2d_host(*_ints(*dims), pm, C.c_int(m), pd, pf))
    else:
        check(lib().dol_sdf_3d_host(*_ints(*dims), pm, C.c_int(m), pd, pf))
    del cells
    return dl, df


# ---- float sites ---------------------------------------------------------------------------------

def init_dirw(mask, dims, out=None, stream=None):
    """InitDirWFromBitMask: direction-weight planes, float32 (4, h, w) for an
    image or (8, d, h, w) for a volume, 1 on set cells and 0 elsewhere."""
    torch = _torch()
    dims = _dims(dims)
    planes = 4 if len(dims) == 2 else 8
    if out is None:
        out = torch.empty((planes,) + tuple(reversed(dims)), dtype=torch.float32, device=mask.device)
    fn = lib().dol_init_dirw_2d if len(dims) == 2 else lib().dol_init_dirw_3d
    check(fn(*_ints(*dims), _ptr(mask), _ptr(out), _stream(stream)))
    return out


def occlusion_sweep(dirw, dims, stream=None):
    """OcclusionSweep in place: quadrant (2D) or octant (3D) occlusion."""
    dims = _dims(dims)
    fn = lib().dol_occlusion_sweep_2d if len(dims) == 2 else lib().dol_occlusion_sweep_3d
    check(fn(*_ints(*dims), _ptr(dirw), _stream(stream)))
    return dirw


def occlusion_sweep_io(dirw_in, dirw_out, dims, stream=None):
    """OcclusionSweep(w, h, d, in, out): the octant occlusion caused by `dirw_in`,
    written to `dirw_out` (each plane's starting cell keeps its value)."""
    dims = _dims(dims)
    if len(dims) != 3:
        raise DolError(ERR_UNSUPPORTED, "the in/out occlusion sweep is 3D, as in the reference")
    check(lib().dol_occlusion_sweep_3d_io(*_ints(*dims), _ptr(dirw_in), _ptr(dirw_out), _stream(stream)))
    return dirw_out


def voxelize(indices, vertices, bbox, dims, mask=None, stream=None):
    """CreateBitMaskFromTriangles: ORs the cells the triangles touch into `mask`
    (int32 words on the device; a zeroed mask by default).  indices: int32
    (t, 3) device tensor or None; vertices: float32 (n, 3) device tensor;
    bbox: six floats (min xyz, max xyz)."""
    torch = _torch()
    w, h, d = _dims(dims)
    if mask is None:
        mask = torch.zeros(mask_words(w, h, d), dtype=torch.int32, device=vertices.device)
    bb = (C.c_float * 6)(*[float(v) for v in bbox])
    tris = int(indices.shape[0]) if indices is not None else int(vertices.shape[0]) // 3
    check(lib().dol_voxelize_triangles(C.c_int(tris), _ptr(indices), _ptr(vertices), bb, *_ints(w, h, d),
                                       _ptr(mask), _stream(stream)))
    return mask


def gen_sites(n, dims, seed):
    """n float sites uniform in continuous cell coordinates, from the reference's
    LCG (24-bit fractions, drawn x, y[, z] per site); float32 array (n, dim)."""
    import numpy as np
    dims = _dims(dims)
    out = np.empty((n, len(dims)), dtype=np.float32)
    s = seed & 0xFFFFFFFF
    for i in range(n):
        for a, extent in enumerate(dims):
            s = (s * 1103515245 + 12345) & 0xFFFFFFFF
            frac = ((s * (1 << 24)) >> 32) / float(1 << 24)
            out[i, a] = np.float32(frac * extent)
    return out


def sites_forward(sites, dims, method="danielsson", stream=None):
    """Distances from every cell centre to its owning site, through a delta
    method run on the cells that hold the sites.  Returns (dist, owner, deltas)."""
    torch = _torch()
    dims = _dims(dims)
    dim = len(dims)
    w, h = dims[0], dims[1]
    d = dims[2] if dim == 3 else 1
    n = int(sites.shape[0])
    mask = torch.empty(mask_words(w, h, d), dtype=torch.int32, device=sites.device)
    cell_site = torch.empty(tuple(reversed(dims)), dtype=torch.int32, device=sites.device)
    check(lib().dol_sites_seed(*_ints(dim, w, h, d, n), _ptr(sites), _ptr(mask), _ptr(cell_site), _stream(stream)))
    deltas = init_deltas(mask, dims, stream=stream)
    propagate(method, deltas, dims, 1, stream=stream)
    owner = torch.empty(tuple(reversed(dims)), dtype=torch.int32, device=sites.device)
    dist = torch.empty(tuple(reversed(dims)), dtype=torch.float32, device=sites.device)
    check(lib().dol_sites_forward(*_ints(dim, w, h, d, n), _ptr(deltas), _ptr(cell_site), _ptr(sites), _ptr(owner),
                                  _ptr(dist), _stream(stream)))
    return dist, owner, deltas


def sites_backward(owner, sites, grad_dist, dims, stream=None):
    """dL/dsites for dL/ddist, with the owner assignment held fixed."""
    torch = _torch()
    dims = _dims(dims)
    dim = len(dims)
    w, h = dims[0], dims[1]
    d = dims[2] if dim == 3 else 1
    n = int(sites.shape[0])
    grad = torch.empty_like(sites)
    check(lib().dol_sites_backward(*_ints(dim, w, h, d, n), _ptr(owner), _ptr(sites), _ptr(grad_dist), _ptr(grad),
                                   None, C.c_size_t(0), _stream(stream)))
    return grad


def site_distance_function():
    """torch.autograd.Function over sites_forward / sites_backward (used for gradient checks)."""
    torch = _torch()

    class SiteDistance(torch.autograd.Function):
        @staticmethod
        def forward(ctx, sites, dims, method):
            s = sites.detach().contiguous()
            dist, owner, _ = sites_forward(s, dims, method)
            ctx.save_for_backward(s, owner)
            ctx.dims = dims
            return dist

        @staticmethod
        def backward(ctx, grad):
            s, owner = ctx.saved_tensors
            return sites_backward(owner, s, grad.contiguous(), ctx.dims), None, None

    return SiteDistance
