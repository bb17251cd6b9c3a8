"""Launch-parameter tuning of fan plans (views per forward-projection CTA,
lines per staged chunk, view split of a single-launch backprojection): every
setting gives the same projections to FP32 rounding, the autotuner returns
settings in range and caches them by shape, and out-of-range requests are
rejected or clamped.

Tolerance: relative L2 <= 1e-6 between settings (the chunked positions round
differently; the sums are otherwise the same)."""
import numpy as np
import pytest

from conftest import rel_l2, small_fan, to_geometry

pytestmark = pytest.mark.gpu

TOL = 1e-6


def _ragged(counts, rng, **kw):
    import torch
    from reconnet_b200.torch_ops import FanPlan
    g = small_fan(**kw)
    angs = np.concatenate([(np.arange(n) * 2 * np.pi / n + 0.003 * n).astype(np.float32) for n in counts])
    plan = FanPlan(to_geometry(g), angs, nbatches=len(counts), nview_per_slice=counts)
    x = torch.from_numpy(rng.random((len(counts), g.nx, g.ny)).astype(np.float32)).cuda()
    return g, plan, x, torch


@pytest.mark.parametrize("siddon", [False, True])
def test_settings_give_the_same_projections(siddon, rng):
    from reconnet_b200 import _native as N
    g, plan, x, torch = _ragged([37, 52], rng)
    bp_type = N.RN_TYPE_SIDDON if siddon else N.RN_TYPE_MATCHED
    p0 = plan.project(x, siddon=siddon)
    y = torch.from_numpy(rng.random(p0.shape).astype(np.float32)).cuda()
    b0 = plan.backproject(y, bp_type)
    plan.set_tuning(99, 10 ** 6, 0)   # clamped: the maxima
    vmax, rmax, _ = plan.tuning()
    assert 1 <= vmax <= 4 and rmax >= 1
    for views, lines, parts in [(1, 1, 2), (2, max(1, rmax // 2), 4), (vmax, rmax, 16), (3, 2, 1)]:
        plan.set_tuning(views, lines, parts)
        v, r, b = plan.tuning()
        assert v == min(views, vmax) and r == min(lines, rmax) and b == parts
        assert rel_l2(plan.project(x, siddon=siddon).cpu().numpy(), p0.cpu().numpy()) <= TOL
        assert rel_l2(plan.backproject(y, bp_type).cpu().numpy(), b0.cpu().numpy()) <= TOL
        plan.check()
    plan.set_tuning(0, 0, 0)   # built-in choices again
    assert torch.equal(plan.project(x, siddon=siddon), p0)


def test_autotune_in_range_cached_and_exact(rng):
    from reconnet_b200 import _native as N
    g, plan, x, torch = _ragged([29, 41, 33], rng, nx=40, ny=36)
    p0 = plan.project(x)
    y = torch.from_numpy(rng.random(p0.shape).astype(np.float32)).cuda()
    b0 = plan.backproject(y, N.RN_TYPE_MATCHED)
    views, lines, parts = plan.autotune(x, N.RN_TYPE_MATCHED)
    assert 1 <= views <= 4 and lines >= 1 and 0 <= parts <= 16
    assert rel_l2(plan.project(x).cpu().numpy(), p0.cpu().numpy()) <= TOL
    assert rel_l2(plan.backproject(y, N.RN_TYPE_MATCHED).cpu().numpy(), b0.cpu().numpy()) <= TOL
    # a second plan of the same shape takes the cached choice
    _, twin, _, _ = _ragged([29, 41, 33], rng, nx=40, ny=36)
    assert twin.autotune(x, N.RN_TYPE_MATCHED) == (views, lines, parts)


def test_out_of_range_settings(rng):
    from reconnet_b200 import _native as N
    g, plan, x, torch = _ragged([20], rng)
    with pytest.raises(N.ReconNetError):
        plan.set_tuning(-1, 0, 0)
    with pytest.raises(N.ReconNetError):
        plan.set_tuning(0, 0, 17)
    plan.set_tuning(99, 10 ** 6, 0)   # clamped to the maxima
    v, r, _ = plan.tuning()
    plan.set_tuning(0, 0, 0)
    v0, r0, _ = plan.tuning()
    assert v <= 4 and r == r0


def test_batched_ossqs_with_and_without_autotune(rng):
    import torch
    from reconnet_b200.ossqs import BatchedOSSQS
    g, plan, x, _ = _ragged([48, 60], rng)
    counts = [48, 60]
    sino = plan.project(x)
    w = torch.ones_like(sino)
    geom = plan.geom
    a = BatchedOSSQS(geom, counts, plan.angles, sino, w, n_subsets=4, autotune=True)
    b = BatchedOSSQS(geom, counts, plan.angles, sino, w, n_subsets=4, autotune=False)
    x0 = torch.zeros_like(x)
    assert rel_l2(a.run(x0, 2).cpu().numpy(), b.run(x0, 2).cpu().numpy()) <= 1e-5


def test_settings_on_a_plan_with_rows_and_channels(rng):
    """A reference-layout plan (2 batches, 3 image slices, 3 detector rows, 2
    channels): the work list spans every (batch, row, channel) slice."""
    import torch
    from reconnet_b200 import _native as N
    from reconnet_b200.torch_ops import FanPlan
    g = small_fan(nz=3, nv=3)
    ang = (np.arange(40) * 2 * np.pi / 40).astype(np.float32)
    plan = FanPlan(to_geometry(g), ang, nbatches=2, nchannels=2)
    x = torch.from_numpy(rng.random(plan.img_shape).astype(np.float32)).cuda()
    p0 = plan.project(x)
    y = torch.from_numpy(rng.random(p0.shape).astype(np.float32)).cuda()
    b0 = plan.backproject(y, N.RN_TYPE_MATCHED)
    for views, lines in [(1, 1), (2, 3), (4, 10 ** 6)]:
        plan.set_tuning(views, lines, 0)
        assert rel_l2(plan.project(x).cpu().numpy(), p0.cpu().numpy()) <= TOL
        assert rel_l2(plan.backproject(y, N.RN_TYPE_MATCHED).cpu().numpy(), b0.cpu().numpy()) <= TOL
    plan.check()
