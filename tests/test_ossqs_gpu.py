"""OS-SQS drivers on the GPU: the graph-captured batched iteration, its parity
with the oracle's subset update, convergence, and the differentiable
unrolled OS-SQS (gradients against central finite differences, eps = 1e-3)."""
import numpy as np
import pytest

from conftest import rel_l2, small_fan, to_geometry

pytestmark = pytest.mark.gpu


def _ragged_problem(rng, counts=(40, 52, 33), noise=False):
    import torch
    from oracle import oracle as O
    g = small_fan()
    angs = [(np.arange(n) * 2 * np.pi / n + 0.05 * s).astype(np.float32) for s, n in enumerate(counts)]
    truth = np.stack([(rng.random((g.nx, g.ny)) * 0.02).astype(np.float32) for _ in counts])
    sinos, ws = [], []
    for s, n in enumerate(counts):
        p = O.fan_fp(truth[s][None, :, :, None, None], angs[s], g, g.nu, 1)[0, :, :, 0, 0]
        w = (0.5 + rng.random(p.shape)).astype(np.float32)
        sinos.append(p.astype(np.float32).ravel())
        ws.append(w.ravel())
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()
    return g, angs, truth, dev(np.concatenate(sinos)), dev(np.concatenate(ws)), sinos, ws


def test_batched_ossqs_graph_matches_eager(rng):
    import torch
    from reconnet_b200.ossqs import BatchedOSSQS
    g, angs, truth, b, w, _, _ = _ragged_problem(rng)
    counts = [a.size for a in angs]
    runs = []
    for graph in (False, True):
        os_ = BatchedOSSQS(to_geometry(g), counts, np.concatenate(angs), b, w, n_subsets=4, beta=0.01,
                           use_graph=graph)
        runs.append(os_.run(torch.zeros((3, g.nx, g.ny), device="cuda"), 2))
        os_.check()
    assert torch.equal(runs[0], runs[1])


@pytest.mark.parametrize("projector", ["dd", "siddon"])
def test_batched_ossqs_iteration_matches_oracle(projector, rng):
    import torch
    from oracle import oracle as O
    from reconnet_b200.ossqs import BatchedOSSQS, interleaved_subsets
    g, angs, truth, b, w, sinos, ws = _ragged_problem(rng)
    counts = [a.size for a in angs]
    M, beta = 3, 0.02
    os_ = BatchedOSSQS(to_geometry(g), counts, np.concatenate(angs), b, w, n_subsets=M, beta=beta, lb=0.0, ub=1.0,
                       projector=projector)
    x0 = (rng.random((3, g.nx, g.ny)) * 0.01).astype(np.float32)
    got = os_.run(torch.from_numpy(x0).cuda(), 1).cpu().numpy()
    for s, n in enumerate(counts):
        sino = sinos[s].reshape(g.nu, n)
        wsn = ws[s].reshape(g.nu, n)
        ones = np.ones((1, g.nx, g.ny, 1, 1), np.float32)
        if projector == "siddon":
            a1 = (O.siddon_fp(ones, angs[s], g, g.nu, 1)[0, :, :, 0, 0] * wsn).astype(np.float32)
            norm = O.siddon_bp(a1[None, :, :, None, None], angs[s], g, (g.nx, g.ny, 1))[0, :, :, 0, 0]
        else:
            a1 = (O.fan_fp(ones, angs[s], g, g.nu, 1)[0, :, :, 0, 0] * wsn).astype(np.float32)
            norm = O.fan_bp(a1[None, :, :, None, None], angs[s], g, (g.nx, g.ny, 1), 2)[0, :, :, 0, 0]
        norm = norm.astype(np.float32)
        x = x0[s]
        for views in interleaved_subsets(n, M):
            x = O.sqs_subset_update(x, sino, wsn, norm, angs[s], views, g, M, beta=beta, lb=0.0,
                                    ub=1.0, projector=projector).astype(np.float32)
        assert rel_l2(got[s], x) <= 1e-4


def test_batched_ossqs_converges(rng):
    import torch
    from reconnet_b200.ossqs import BatchedOSSQS
    g, angs, truth, b, w, _, _ = _ragged_problem(rng)
    counts = [a.size for a in angs]
    os_ = BatchedOSSQS(to_geometry(g), counts, np.concatenate(angs), b, w, n_subsets=4)
    x = torch.zeros((3, g.nx, g.ny), device="cuda")
    t = torch.from_numpy(truth).cuda()
    e0 = float((x - t).norm())
    errs = [float((os_.run(x, k) - t).norm()) for k in (2, 8)]
    assert errs[0] < 0.7 * e0 and errs[1] < errs[0]


def _unrolled_setup(rng, B=2, M=2, K=3):
    import torch
    from oracle import oracle as O
    from reconnet_b200.torch_ops import FanPlan
    g = small_fan(nx=32, ny=28, nu=48, da=0.0035)
    nview = 24
    ang = (np.arange(nview) * 2 * np.pi / nview).astype(np.float32)
    truth = (rng.random((B, g.nx, g.ny, 1, 1)) * 0.02).astype(np.float32)
    sino = O.fan_fp(truth, ang, g, g.nu, 1).astype(np.float32)
    w = (0.5 + rng.random(sino.shape)).astype(np.float32)
    geom = to_geometry(g)
    full = FanPlan(geom, ang, nbatches=B)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()
    wd = dev(w)
    norm = full.backproject(full.project(torch.ones(full.img_shape, device="cuda")) * wd, 2)
    plans, bs, ws = [], [], []
    for m in range(M):
        v = np.arange(m, nview, M)
        plans.append(FanPlan(geom, ang[v], nbatches=B))
        bs.append(dev(sino[:, :, v]))
        ws.append(dev(w[:, :, v]))
    return plans, bs, ws, norm, dev(truth), K


def test_unrolled_ossqs_gradients_match_finite_differences(rng):
    import torch
    from reconnet_b200.ossqs import unrolled_ossqs
    plans, bs, ws, norm, truth, K = _unrolled_setup(rng)
    x0 = torch.zeros_like(truth)

    def loss(step, tvw, x_init=x0, checkpoint=True):
        x = unrolled_ossqs(x_init, plans, bs, ws, norm, step, tvw, checkpoint=checkpoint)
        return ((x - truth).double() ** 2).sum()

    step = torch.tensor([0.8, 0.9, 1.0], device="cuda", requires_grad=True)
    tvw = torch.tensor([0.02, 0.01, 0.005], device="cuda", requires_grad=True)
    L = loss(step, tvw)
    gs, gt = torch.autograd.grad(L, (step, tvw))
    # checkpointing does not change the gradient
    gs2, gt2 = torch.autograd.grad(loss(step, tvw, checkpoint=False), (step, tvw))
    assert torch.allclose(gs, gs2, rtol=1e-5, atol=1e-9) and torch.allclose(gt, gt2, rtol=1e-5, atol=1e-9)
    eps = 1e-3
    with torch.no_grad():
        for vec, grad, other, first in ((step, gs, tvw, True), (tvw, gt, step, False)):
            for i in range(K):
                d = torch.zeros_like(vec)
                d[i] = eps
                lp = loss(vec + d, other) if first else loss(other, vec + d)
                lm = loss(vec - d, other) if first else loss(other, vec - d)
                fd = float(lp - lm) / (2 * eps)
                assert abs(fd - float(grad[i])) <= 2e-2 * abs(fd) + 1e-7, (first, i, fd, float(grad[i]))
    # directional derivative w.r.t. the starting image
    x_init = (0.01 * torch.rand_like(truth)).requires_grad_(True)
    gx, = torch.autograd.grad(loss(step.detach(), tvw.detach(), x_init), (x_init,))
    # a step along the gradient (a random direction is nearly orthogonal to it),
    # 1e-5 at most per pixel: well inside the TV smoothing scale sqrt(1e-6)
    v = gx / gx.abs().max() * 1e-5
    with torch.no_grad():
        fd = float(loss(step, tvw, x_init + v) - loss(step, tvw, x_init - v)) / 2
    assert abs(fd - float((gx * v).sum())) <= 2e-2 * abs(fd)
