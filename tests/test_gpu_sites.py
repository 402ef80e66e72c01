"""Distances to float sites and their gradient.

Forward: the delta method's deltas are bit-exact to the oracle on the seeded
mask, the owner of every cell is the site held by the cell its delta reaches,
and d = |p - site| equals an fp32 recomputation.  Backward: against an FP64
brute-force gradient over the same (fixed) owner assignment, max relative
error <= 1e-5; against central finite differences (h = 1e-3 cell) of the FP64
loss for sites that stay in their cell, relative error <= 1e-4.  The loss is
sum (d - d_t)^2 with d_t the field of the same sites jittered by N(0, 0.5)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [((512, 512), 4096, "danielsson"), ((512, 512), 4096, "jumpflood"),
         ((128, 128, 128), 4096, "danielsson"), ((64, 48, 40), 500, "jumpflood")]


def _centres(dims):
    grids = np.meshgrid(*[np.arange(n, dtype=np.float64) + 0.5 for n in reversed(dims)], indexing="ij")
    return [g for g in reversed(grids)]   # x, y[, z], each shaped (d, h, w) / (h, w)


def _setup(dol, torch, dims, n, method):
    sites = dol.gen_sites(n, dims, 11)
    rng = np.random.default_rng(11)
    jit = (sites + rng.normal(0, 0.5, sites.shape)).astype(np.float32)
    jit = np.clip(jit, 0, np.array(dims, np.float32) - 1e-3).astype(np.float32)
    s = torch.from_numpy(sites).cuda()
    dist, owner, deltas = dol.sites_forward(s, dims, method)
    dt, _, _ = dol.sites_forward(torch.from_numpy(jit).cuda(), dims, method)
    dol.sync()
    return sites, s, dist, owner, deltas, dt


@pytest.mark.parametrize("dims,n,method", CASES)
def test_sites_forward(dol, O, cuda, dims, n, method):
    torch = cuda
    sites, s, dist, owner, deltas, _ = _setup(dol, torch, dims, n, method)
    # seeded mask: the cells holding the sites
    cells = np.floor(sites).astype(np.int64)
    b = np.zeros(tuple(reversed(dims)), bool)
    b[tuple(cells[:, a] for a in reversed(range(len(dims))))] = True
    m = O.bool_to_mask(b)
    want = O.propagate(method, O.init_deltas(m, dims), dims, 1)
    np.testing.assert_array_equal(deltas.cpu().numpy(), want)
    own = owner.cpu().numpy()
    assert (own >= 0).all()
    # the owner sits in the cell the delta points at, smallest index on ties
    cen = _centres(dims)
    tgt = [np.floor(c).astype(np.int64) + want[..., a] for a, c in enumerate(cen)]
    np.testing.assert_array_equal(cells[own.reshape(-1)].T, np.stack([t.reshape(-1) for t in tgt]))
    # fp32 distance, same operation order (no fused multiply-add)
    e = [(sites[own][..., a] - cen[a].astype(np.float32)).astype(np.float32) for a in range(len(dims))]
    s2 = e[0] * e[0] + e[1] * e[1]
    if len(dims) == 3:
        s2 = (s2 + e[2] * e[2]).astype(np.float32)
    np.testing.assert_array_equal(dist.cpu().numpy(), np.sqrt(s2.astype(np.float32)))


def _ref_grad(sites, own, gd, dims):
    cen = _centres(dims)
    e = np.stack([sites[own][..., a].astype(np.float64) - cen[a] for a in range(len(dims))], axis=-1)
    ln = np.sqrt((e * e).sum(-1))
    contrib = (gd.astype(np.float64) / ln)[..., None] * e
    g = np.zeros((sites.shape[0], len(dims)), np.float64)
    np.add.at(g, own.reshape(-1), contrib.reshape(-1, len(dims)))
    return g


@pytest.mark.parametrize("dims,n,method", CASES)
def test_sites_backward_against_fp64_and_fd(dol, O, cuda, dims, n, method):
    torch = cuda
    sites, s, dist, owner, deltas, dt = _setup(dol, torch, dims, n, method)
    grad_d = (2.0 * (dist - dt)).contiguous()
    g = dol.sites_backward(owner, s, grad_d, dims).cpu().numpy().astype(np.float64)
    own = owner.cpu().numpy()
    ref = _ref_grad(sites, own, grad_d.cpu().numpy(), dims)
    scale = np.linalg.norm(ref, axis=1)
    sel = scale > 1e-6 * scale.max()
    rel = np.linalg.norm(g - ref, axis=1)[sel] / scale[sel]
    assert rel.max() <= 1e-5, rel.max()

    # central finite differences of the FP64 loss with the owner assignment held fixed
    cen = _centres(dims)
    dtn = dt.cpu().numpy().astype(np.float64)
    rng = np.random.default_rng(3)
    h = 1e-3
    picked = [k for k in rng.permutation(n)[:60]
              if np.all(np.floor(sites[k] - h) == np.floor(sites[k] + h))]
    flat_own = own.reshape(-1)
    for k in picked:
        cellsk = np.nonzero(flat_own == k)[0]
        if len(cellsk) == 0:
            continue
        pc = [c.reshape(-1)[cellsk] for c in cen]
        tgt = dtn.reshape(-1)[cellsk]

        def loss(sk):
            dd = np.sqrt(sum((sk[a] - pc[a]) ** 2 for a in range(len(dims))))
            return ((dd - tgt) ** 2).sum()
        fd = np.zeros(len(dims))
        for a in range(len(dims)):
            sp = sites[k].astype(np.float64).copy()
            sm = sp.copy()
            sp[a] += h
            sm[a] -= h
            fd[a] = (loss(sp) - loss(sm)) / (2 * h)
        # analytic gradient of the same FP64 loss
        dd = np.sqrt(sum((sites[k][a] - pc[a]) ** 2 for a in range(len(dims))))
        an = np.array([(2 * (dd - tgt) * (sites[k][a] - pc[a]) / dd).sum() for a in range(len(dims))])
        assert np.linalg.norm(fd - an) <= 1e-4 * max(np.linalg.norm(an), 1e-3), (k, fd, an)
        # the kernel's gradient for this site agrees with the analytic one
        assert np.linalg.norm(g[k] - an) <= 1e-4 * max(np.linalg.norm(an), 1e-2), (k, g[k], an)


def test_autograd_function(dol, cuda):
    torch = cuda
    dims = (96, 80)
    sites = torch.from_numpy(dol.gen_sites(300, dims, 11)).cuda().requires_grad_(True)
    F = dol.site_distance_function()
    d = F.apply(sites, dims, "danielsson")
    target = d.detach() * 0.9
    loss = ((d - target) ** 2).sum()
    (g,) = torch.autograd.grad(loss, sites)
    _, owner, _ = dol.sites_forward(sites.detach(), dims, "danielsson")
    want = dol.sites_backward(owner, sites.detach(), (2 * (d - target)).detach().contiguous(), dims)
    assert torch.equal(g, want)
