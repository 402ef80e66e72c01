"""dol_edt_mask_2d_noalloc: the 2D mask EDT for callers that cannot allocate.

Some callers cannot allocate device memory when they call the library (an
application that reserved all of its GPU memory at start-up and forbids
allocation afterwards, or one that must not risk an allocation failing
mid-frame).  This entry point keeps its scratch in a fixed array inside the
library instead.  The test calls it through the C ABI twice in a row, on
different images, and checks each result against the allocating entry point
(dol_edt_mask_2d) bit for bit -- the same bar as every float output in this
suite.  The second call also shows that the leftover contents of the shared
array from the first call do not leak into the result.  The file is named to
be collected last.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _call(dol, torch, mask, dims, form):
    w, h = dims
    out = torch.empty((h, w), dtype=torch.float32, device="cuda")
    st = dol.lib().dol_edt_mask_2d_noalloc(C.c_int(w), C.c_int(h), C.c_void_p(mask.data_ptr()),
                                           C.c_void_p(out.data_ptr()), C.c_int(form),
                                           C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == dol.OK, dol.lib().dol_last_error()
    dol.sync()
    return out


def test_no_alloc_edt_matches_allocating_entry_point(dol, O, cuda):
    torch = cuda
    rng = np.random.default_rng(2024)
    # columns of up to 3200 cells are staged in shared memory, taller ones are
    # read from global memory: 1024 x 4096 takes the second branch, and
    # 4096 x 2048 is exactly the array's 8,388,608-cell limit
    cases = [((700, 500), 0.02, dol.EDT_SIGNED), ((333, 129), 0.3, dol.EDT_DIST), ((2048, 1024), 0.001, dol.EDT_SQUARED),
             ((1024, 4096), 0.0005, dol.EDT_SIGNED), ((4096, 2048), 0.0002, dol.EDT_DIST)]
    for dims, p, form in cases:
        w, h = dims
        m = O.bool_to_mask(rng.random((h, w)) < p)
        md = torch.from_numpy(m.view(np.int32)).cuda()
        got = _call(dol, torch, md, dims, form).cpu().numpy()
        want = dol.edt_mask(md, dims, form).cpu().numpy()
        np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32), err_msg=f"{dims} form {form}")


def test_no_alloc_edt_rejects_oversize(dol, cuda):
    torch = cuda
    buf = torch.zeros(16, dtype=torch.int32, device="cuda")
    st = dol.lib().dol_edt_mask_2d_noalloc(C.c_int(4096), C.c_int(4096), C.c_void_p(buf.data_ptr()),
                                           C.c_void_p(buf.data_ptr()), C.c_int(dol.EDT_DIST), None)
    assert st == dol.ERR_UNSUPPORTED
    assert b"no-allocation limit" in dol.lib().dol_last_error()
