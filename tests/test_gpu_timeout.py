"""Failure detection: a bounded device-side wait that runs out is reported.

Every spin-wait in the library's kernels has an iteration limit; when it runs
out the kernel records the failure in a mapped host word, stops waiting and
finishes its launch, and the next dol_sync() on the stream returns
DOL_ERR_TIMEOUT.  The reference has no failure detection to match (asserts
only, DistanceOcclusionLib.cpp:14-18).

The test hook dol_test_wait_hooks makes one sweep of the 3D FastSweep
wavefront wait for a row flag that no row ever writes (a plain global-memory
flag, polled with a short limit), so every row wait of that sweep gives up.
Nothing faults or traps: the launch ends on its own, the call reports the
timeout, and a normal call on the same stream afterwards succeeds with the
reference's deltas.
"""
import ctypes as C
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("stall_sweep", [0, 5])
def test_fastsweep3_wait_runs_out_then_stream_recovers(dol, O, cuda, stall_sweep):
    torch = cuda
    L = dol.lib()
    dims = (24, 12, 10)
    rng = np.random.default_rng(31 + stall_sweep)
    mask = O.bool_to_mask(rng.random((dims[2], dims[1], dims[0])) < 0.1)
    md = torch.from_numpy(mask.view(np.int32)).cuda()
    bor = dol.init_border(md, dims)
    sp = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert L.dol_sync(sp) == dol.OK

    work = bor.clone()
    L.dol_test_wait_hooks(C.c_int(stall_sweep), C.c_uint(2000))
    try:
        t0 = time.perf_counter()
        dol.fastsweep(work, dims, 2)            # queued: nothing is known yet
        rc = L.dol_sync(sp)
        elapsed = time.perf_counter() - t0
    finally:
        L.dol_test_wait_hooks(C.c_int(-1), C.c_uint(0))
    assert rc == dol.ERR_TIMEOUT, L.dol_last_error()
    assert b"gave up" in L.dol_last_error()
    assert elapsed < 60.0

    # the error word is cleared by the sync that reported it; the stream and
    # the context stay usable and give the reference's result
    work2 = bor.clone()
    dol.fastsweep(work2, dims, 2)
    assert L.dol_sync(sp) == dol.OK, L.dol_last_error()
    want = O.propagate("fastsweep", O.border_init(mask, dims), dims, 2)
    np.testing.assert_array_equal(work2.cpu().numpy(), want)
