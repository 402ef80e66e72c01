"""The GPU mesh voxeliser against the reference's CreateBitMaskFromTriangles.

dol_voxelize_triangles must set exactly the reference's bits
(MeshSupport.cpp:369-475): on the reference's sample mesh (data/plant2.obj as
the reference's own OBJ reader sees it, dumped at build time into
oracle/_ref/plant2.tri) at the tool's default volume size and others, and on
synthetic triangle soups with tiny, large and degenerate triangles.  The
oracle's restatement is pinned to the reference in test_oracle_pin.py; the
reference build itself is compared too where present.  The mask then feeds the
distance transforms on the device.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TRI = os.path.join(ROOT, "oracle", "_ref", "plant2.tri")


def _cases(O, rng, synthetic=True):
    cases = []
    if synthetic:
        cases = [("soup", O.random_triangles(rng, 3000)), ("big", O.random_triangles(rng, 40, scale=(0.5, 2.0)))]
    if os.path.exists(TRI):
        cases.append(("plant2", O.load_tri(TRI)))
    return cases


@pytest.mark.parametrize("dims", [(32, 32, 32), (64, 64, 64), (100, 80, 60), (33, 17, 70), (256, 256, 256)])
def test_voxelize_matches_reference(dol, O, cuda, dims):
    torch = cuda
    rng = np.random.default_rng(sum(dims) + 3)
    for name, (idx, v, bb) in _cases(O, rng):
        got = dol.voxelize(torch.from_numpy(idx).cuda(), torch.from_numpy(v).cuda(), bb, dims).cpu().numpy()
        want = O.voxelize(idx, v, bb, dims, use_ref=O.ref() is not None)
        np.testing.assert_array_equal(got.view(np.uint32), want, err_msg=f"{name} {dims}")
        # ORed into an existing mask; without indices (vertices three per triangle)
        prior = O.bool_to_mask(rng.random(tuple(reversed(dims))) < 0.02)
        flat = np.ascontiguousarray(v[idx.reshape(-1)])
        got = dol.voxelize(None, torch.from_numpy(flat).cuda(), bb, dims,
                           mask=torch.from_numpy(prior.view(np.int32).copy()).cuda()).cpu().numpy()
        np.testing.assert_array_equal(got.view(np.uint32), O.voxelize(idx, v, bb, dims, mask=prior), err_msg=name)


def test_voxelized_mask_feeds_the_distance_field(dol, O, cuda):
    """Voxelise on the device, then the signed Danielsson field of that mask,
    with no host round trip: equal to the oracle on the same mask."""
    if not os.path.exists(TRI):
        pytest.skip("plant2.tri not built")
    torch = cuda
    dims = (64, 64, 64)
    idx, v, bb = O.load_tri(TRI)
    md = dol.voxelize(torch.from_numpy(idx).cuda(), torch.from_numpy(v).cuda(), bb, dims)
    dl, df = dol.sdf(md, dims, "danielsson")
    m = md.cpu().numpy().view(np.uint32)
    want = O.propagate("danielsson", O.border_init(m, dims), dims, 2)
    np.testing.assert_array_equal(dl.cpu().numpy(), want)


def test_voxelize_rejects_bad_boxes(dol, cuda):
    torch = cuda
    v = torch.zeros((3, 3), dtype=torch.float32, device="cuda")
    for bb in ([0, 0, 0, 1, 1, 0], [0, 0, 0, 1, float("nan"), 1], [1, 0, 0, 0, 1, 1]):
        with pytest.raises(dol.DolError):
            dol.voxelize(None, v, bb, (8, 8, 8))
