"""Batched signed fields (one persistent launch over many uneven masks and
volumes) against the oracle and against per-item calls; the CUDA-graph replay
gives the same bytes; the batch generator rasterises the same bits on host
and device."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def gen_batch(dol, torch, n2, n3, seed):
    L = dol.lib()
    n = n2 + n3
    items = (ItemArray(dol) * n)()
    tw, tb, tc = C.c_longlong(), C.c_longlong(), C.c_longlong()
    dol.check(L.dol_gen_batch(n2, n3, C.c_uint32(seed), items, C.byref(tw), C.byref(tb), C.byref(tc), None, None))
    masks = torch.empty(tw.value, dtype=torch.int32, device="cuda")
    dol.check(L.dol_gen_batch(n2, n3, C.c_uint32(seed), items, None, None, None, C.c_void_p(masks.data_ptr()),
                              C.c_void_p(torch.cuda.current_stream().cuda_stream)))
    return items, masks, tb.value, tc.value


_ITEM = None


def ItemArray(dol):
    global _ITEM
    if _ITEM is None:
        class Item(C.Structure):
            _fields_ = [("w", C.c_int), ("h", C.c_int), ("d", C.c_int), ("reserved", C.c_int),
                        ("mask_word_offset", C.c_longlong), ("delta_byte_offset", C.c_longlong),
                        ("dist_offset", C.c_longlong)]
        _ITEM = Item
    return _ITEM


def test_batch_generator_host_equals_device(dol, cuda):
    torch = cuda
    items, masks, _, _ = gen_batch(dol, torch, 30, 3, 99)
    host = np.zeros(masks.numel(), np.uint32)
    dol.lib().dol_gen_batch_host(30, 3, C.c_uint32(99), host.ctypes.data_as(C.c_void_p))
    np.testing.assert_array_equal(masks.cpu().numpy().view(np.uint32), host)
    assert host.any()


def test_batch_matches_oracle_and_per_item_calls(dol, O, cuda):
    torch = cuda
    L = dol.lib()
    n2, n3 = 48, 4
    items, masks, dbytes, cells = gen_batch(dol, torch, n2, n3, 5)
    n = n2 + n3
    deltas = torch.zeros(dbytes, dtype=torch.uint8, device="cuda")
    dist = torch.zeros(cells, dtype=torch.float32, device="cuda")
    sp = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    dol.check(L.dol_batch_sdf(n, items, C.c_void_p(masks.data_ptr()), C.c_void_p(deltas.data_ptr()),
                              C.c_void_p(dist.data_ptr()), None, C.c_size_t(0), sp))
    dol.sync()
    mh = masks.cpu().numpy().view(np.uint32)
    dh = deltas.cpu().numpy()
    fh = dist.cpu().numpy()
    for i in range(n):
        it = items[i]
        dims = (it.w, it.h) if it.d == 1 else (it.w, it.h, it.d)
        nw = O.mask_words(*dims)
        m = mh[it.mask_word_offset: it.mask_word_offset + nw].copy()
        cells_i = it.w * it.h * it.d
        want = O.propagate("danielsson", O.border_init(m, dims), dims, 2)
        cb = 4 if it.d == 1 else 6
        got = dh[it.delta_byte_offset: it.delta_byte_offset + cells_i * cb].view(np.int16).reshape(want.shape)
        np.testing.assert_array_equal(got, want, err_msg=f"item {i} dims {dims}")
        wd = O.deltas_to_dist(want, dims, 2, m)
        gd = fh[it.dist_offset: it.dist_offset + cells_i].reshape(wd.shape)
        np.testing.assert_array_equal(gd.view(np.uint32), wd.view(np.uint32), err_msg=f"item {i}")
        if i % 13 == 0:   # the per-item one-call path gives the same bytes
            md = torch.from_numpy(m.view(np.int32)).cuda()
            dl, df = dol.sdf(md, dims, "danielsson")
            np.testing.assert_array_equal(dl.cpu().numpy(), want)


def test_batch_graph_replay(dol, cuda):
    torch = cuda
    L = dol.lib()
    n2, n3 = 20, 2
    items, masks, dbytes, cells = gen_batch(dol, torch, n2, n3, 8)
    n = n2 + n3
    ws_bytes = L.dol_batch_workspace_size(n)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device="cuda")
    sp = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    d1 = torch.zeros(dbytes, dtype=torch.uint8, device="cuda")
    f1 = torch.zeros(cells, dtype=torch.float32, device="cuda")
    dol.check(L.dol_batch_prepare(n, items, C.c_void_p(ws.data_ptr()), C.c_size_t(ws_bytes), sp))
    dol.check(L.dol_batch_run(n, C.c_void_p(masks.data_ptr()), C.c_void_p(d1.data_ptr()), C.c_void_p(f1.data_ptr()),
                              C.c_void_p(ws.data_ptr()), sp))
    dol.sync()
    d2 = torch.zeros_like(d1)
    f2 = torch.zeros_like(f1)
    g = C.c_void_p()
    dol.check(L.dol_batch_graph_create(n, C.c_void_p(masks.data_ptr()), C.c_void_p(d2.data_ptr()),
                                       C.c_void_p(f2.data_ptr()), C.c_void_p(ws.data_ptr()), C.byref(g)))
    for _ in range(2):
        dol.check(L.dol_graph_launch(g, sp))
    dol.sync()
    L.dol_graph_destroy(g)
    assert torch.equal(d1, d2) and torch.equal(f1, f2)


@pytest.mark.parametrize("shapes", [
    [(40, 30, 20)],                                                    # one narrow volume only
    [(300, 9, 5), (20, 30, 1), (64, 10, 12)],                          # a wide volume (whole CTA), an image, a volume
    [(600, 40, 1), (33, 7, 9), (50, 20, 3), (100, 100, 1), (257, 3, 1)],
    [(16, 8, 4)] * 40 + [(512, 64, 1)],                                # many small volumes, one wide image
])
def test_batch_queue_mixes(dol, O, cuda, shapes):
    """Every mix of the two queues (narrow volumes one per warp; wide items per
    CTA, then narrow images) gives the oracle's bytes for every item."""
    torch = cuda
    L = dol.lib()
    rng = np.random.default_rng(len(shapes) * 7 + shapes[0][0])
    Item = ItemArray(dol)
    items = (Item * len(shapes))()
    masks, mo, do, fo = [], 0, 0, 0
    for i, (w, h, d) in enumerate(shapes):
        dims = (w, h) if d == 1 else (w, h, d)
        m = O.bool_to_mask(rng.random(tuple(reversed(dims))) < 0.08)
        masks.append((dims, m))
        items[i] = Item(w, h, d, 0, mo, do, fo)
        mo += m.size
        do += (w * h * d * (4 if d == 1 else 6) + 15) // 16 * 16   # item regions 16-byte aligned
        fo += w * h * d
    mflat = np.concatenate([m for _, m in masks]).astype(np.uint32)
    md = torch.from_numpy(mflat.view(np.int32)).cuda()
    deltas = torch.zeros(do, dtype=torch.uint8, device="cuda")
    dist = torch.zeros(fo, dtype=torch.float32, device="cuda")
    sp = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    dol.check(L.dol_batch_sdf(len(shapes), items, C.c_void_p(md.data_ptr()), C.c_void_p(deltas.data_ptr()),
                              C.c_void_p(dist.data_ptr()), None, C.c_size_t(0), sp))
    dol.sync()
    dh, fh = deltas.cpu().numpy(), dist.cpu().numpy()
    for i, (dims, m) in enumerate(masks):
        it = items[i]
        want = O.propagate("danielsson", O.border_init(m, dims), dims, 2)
        cells = it.w * it.h * it.d
        cb = 4 if it.d == 1 else 6
        got = dh[it.delta_byte_offset: it.delta_byte_offset + cells * cb].view(np.int16).reshape(want.shape)
        np.testing.assert_array_equal(got, want, err_msg=f"item {i} dims {dims}")
        wd = O.deltas_to_dist(want, dims, 2, m)
        gd = fh[it.dist_offset: it.dist_offset + cells].reshape(wd.shape)
        np.testing.assert_array_equal(gd.view(np.uint32), wd.view(np.uint32), err_msg=f"item {i}")


def test_batch_rejects_misaligned_offsets(dol, cuda):
    """A 2D item whose cells would not start on a 4-byte boundary is refused
    before anything launches."""
    torch = cuda
    L = dol.lib()
    Item = ItemArray(dol)
    items = (Item * 2)()
    items[0] = Item(33, 7, 9, 0, 0, 0, 0)                      # 3D, 33*7*9*6 = 12474 bytes
    items[1] = Item(20, 30, 1, 0, 9 * 7 * 2, 12474, 33 * 7 * 9)   # 2D at an offset that is 2 mod 4
    ws_bytes = L.dol_batch_workspace_size(2)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device="cuda")
    st = L.dol_batch_prepare(2, items, C.c_void_p(ws.data_ptr()), C.c_size_t(ws_bytes), None)
    assert st == dol.ERR_INVALID_ARG
    assert b"multiple of 4" in L.dol_last_error()
