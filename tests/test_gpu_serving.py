"""Serving: incremental re-sort and continuous batching give exactly the per-call results.

* A batch built with a linear-cell hint (points in a previous cell order, each with its previous
  cell) must equal the full build of the same input, whether the hint holds (the incremental path
  runs) or not (the device falls back to the full sort).
* Every request of the search server must return the same pair set whether it ran alone or batched
  with others, and the same as radiusSearch on the scene's positions.
"""
import numpy as np
import pytest
import torch

import cases

pytestmark = pytest.mark.gpu


def _cloud(seed, n, dim=3, periodic=True):
    g = torch.Generator().manual_seed(seed)
    x = torch.rand(n, dim, generator=g) * 2 - 1
    dx = 2.0 / n ** (1.0 / dim)
    h = (3 * 50 * dx ** 3 / (4 * np.pi)) ** (1 / 3) if dim == 3 else (32 * dx * dx / np.pi) ** 0.5
    return x, torch.full((n,), float(h)), h


def _table(xs, hs, per):
    from torchcompactradius_b200 import batched
    t = batched.cloud_table(len(xs))
    for k, (x, h) in enumerate(zip(xs, hs)):
        d = x.shape[1]
        t["dim"][k] = d
        t["periodic_mask"][k] = (1 << d) - 1 if per else 0
        t["domain_min"][k, :d] = -1.0
        t["domain_max"][k, :d] = 1.0
        t["n_query"][k] = t["n_ref"][k] = x.shape[0]
        t["query_pos"][k] = t["ref_pos"][k] = x.data_ptr()
        t["query_sup"][k] = t["ref_sup"][k] = h.data_ptr()
    return t


def _run(xs, hs, per, hint=None, want_order=False):
    from torchcompactradius_b200 import batched
    dev = torch.device("cuda")
    n = sum(x.shape[0] for x in xs)
    lin_out = torch.empty(n, dtype=torch.int32, device=dev)
    order = torch.empty(n, dtype=torch.int32, device=dev)
    out = batched.run_batch(_table(xs, hs, per), "gather", True, "csr", dev, lin_hint=hint, lin_out=lin_out,
                            order_out=order)
    return out, lin_out, order


@pytest.mark.parametrize("per", [True, False])
def test_incremental_build_equals_full_build(per):
    xs, hs = [], []
    for k, n in enumerate((30000, 4000, 120000)):
        x, h, hv = _cloud(k, n)
        xs.append(x.cuda())
        hs.append(h.cuda())
    _, lin, order = _run(xs, hs, per)
    # put every cloud in its cell order and move its points a little
    base = 0
    moved_x = []
    for k, x in enumerate(xs):
        n = x.shape[0]
        perm = (order[base:base + n] - base).long()
        g = torch.Generator(device="cuda").manual_seed(100 + k)
        d = torch.randn(x.shape, generator=g, device="cuda") * 0.05 * float(hs[k][0])
        moved_x.append((x.index_select(0, perm) + d).contiguous())
        hs[k] = hs[k].index_select(0, perm).contiguous()
        base += n
    full, lin_full, order_full = _run(moved_x, hs, per)
    inc, lin_inc, order_inc = _run(moved_x, hs, per, hint=lin)
    assert int(inc["info"][7]) > 0, "the incremental path did not run"
    assert int(full["info"][7]) == -2
    assert torch.equal(full["offsets"], inc["offsets"])
    assert torch.equal(full["col"], inc["col"])
    assert torch.equal(order_full, order_inc) and torch.equal(lin_full, lin_inc)
    # a hint that does not hold: the device falls back to the full sort, same result
    bad = lin[torch.randperm(lin.numel(), device="cuda")]
    fb, _, order_fb = _run(moved_x, hs, per, hint=bad)
    assert int(fb["info"][7]) == -1
    assert torch.equal(full["col"], fb["col"]) and torch.equal(order_full, order_fb)


def _scene_inputs(n_scenes=6, seed=7):
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n_scenes):
        n = int(np.exp(rng.uniform(np.log(2000), np.log(60000))))
        x, h, hv = _cloud(1000 + k, n)
        out.append((x, h, hv))
    return out


def _displacements(scene_inputs, steps):
    """Deterministic displacements per (scene, step), user order."""
    d = {}
    for k, (x, h, hv) in enumerate(scene_inputs):
        for s in range(steps):
            g = torch.Generator().manual_seed(10000 * k + s)
            d[k, s] = torch.randn(x.shape, generator=g) * 0.05 * hv
    return d


def _serve(scene_inputs, disp, steps, together):
    import torchcompactradius_b200 as tcr
    from torchcompactradius_b200.serving import Request, Scene, SearchServer
    dom = tcr.DomainDescription(torch.full((3,), -1.0), torch.full((3,), 1.0), torch.tensor([True] * 3), 3)
    srv = SearchServer(hbm_budget=4e9, slots=2)
    for x, h, hv in scene_inputs:
        srv.add_scene(Scene(x.cuda(), h.cuda(), dom))
    res = {}
    with srv:
        if together:
            reqs = []
            for s in range(steps):
                for k in range(len(scene_inputs)):
                    reqs.append(((k, s), srv.submit(Request(k, disp[k, s].cuda()))))
            for key, r in reqs:
                res[key] = r.wait(120)
        else:
            for s in range(steps):
                for k in range(len(scene_inputs)):
                    res[k, s] = srv.search(k, disp[k, s].cuda(), timeout=120)
    return res, srv


def test_server_results_are_the_same_alone_and_in_the_mix():
    import torchcompactradius_b200 as tcr
    steps = 3
    scenes = _scene_inputs()
    disp = _displacements(scenes, steps)
    alone, _ = _serve(scenes, disp, steps, together=False)
    mixed, srv = _serve(scenes, disp, steps, together=True)
    assert srv.batched_requests == steps * len(scenes)
    assert srv.batches < srv.batched_requests  # requests were batched together
    dom = tcr.DomainDescription(torch.full((3,), -1.0), torch.full((3,), 1.0), torch.tensor([True] * 3), 3)
    for k, (x, h, hv) in enumerate(scenes):
        pos = x.cuda()
        for s in range(steps):
            pos = pos + disp[k, s].cuda()
            a = cases.canonical(alone[k, s].row.cpu().numpy(), alone[k, s].col.cpu().numpy())
            b = cases.canonical(mixed[k, s].row.cpu().numpy(), mixed[k, s].col.cpu().numpy())
            np.testing.assert_array_equal(a, b)
            ref = tcr.radiusSearch(tcr.PointCloud(pos, h.cuda()), mode="gather", domain=dom, algorithm="compact")
            c = cases.canonical(ref.row.cpu().numpy(), ref.col.cpu().numpy())
            np.testing.assert_array_equal(a, c)
