"""Siddon cone-beam pair with arbitrary per-view geometry (SiddonCone.cu) on
the GPU: forward projection and its transpose against the FP64 oracle (exact
crossings), the adjoint identity, the reference-named host entry points,
and the cone OS-SQS loop (ossqs.cu:163-333) against the oracle's.

Tolerance: relative L2 <= 1e-5 against the FP64 oracle; |<Ax,y> - <x,A^T y>|
/ |<Ax,y>| <= 1e-5."""
import os
import sys
from types import SimpleNamespace as NS

import numpy as np
import pytest

from conftest import ROOT, rel_l2

sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
import make_golden as M  # noqa: E402

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _case(name, B=1, C=1):
    import torch
    from reconnet_b200.torch_ops import ConeGeometry, ConePlan
    g, dc, du, dv, src = M.cone_geometry(name)
    plan = ConePlan(ConeGeometry(**g), dc, du, dv, src, nbatches=B, nchannels=C)
    return NS(**g), (dc, du, dv, src), plan, torch


@pytest.mark.parametrize("name", M.CONE_CASES)
def test_cone_fp_matches_oracle(name, rng):
    from oracle import oracle as O
    g, geo, plan, torch = _case(name)
    x = rng.random(plan.img_shape).astype(np.float32)
    got = plan.project(torch.from_numpy(x).cuda()).cpu().numpy()
    assert rel_l2(got, O.cone_fp(x, *geo, g, g.nu, g.nv)) <= TOL


@pytest.mark.parametrize("name", M.CONE_CASES)
def test_cone_bp_matches_oracle(name, rng):
    from oracle import oracle as O
    g, geo, plan, torch = _case(name)
    y = rng.random(plan.prj_shape).astype(np.float32)
    got = plan.backproject(torch.from_numpy(y).cuda()).cpu().numpy()
    assert rel_l2(got, O.cone_bp(y, *geo, g, (g.nx, g.ny, g.nz))) <= TOL


@pytest.mark.parametrize("name", M.CONE_CASES)
def test_cone_adjoint(name, rng):
    g, geo, plan, torch = _case(name, B=2, C=2)
    x = torch.from_numpy(rng.random(plan.img_shape).astype(np.float32)).cuda()
    y = torch.from_numpy(rng.random(plan.prj_shape).astype(np.float32)).cuda()
    ax = plan.project(x).double()
    aty = plan.backproject(y).double()
    lhs, rhs = float((ax * y.double()).sum()), float((x.double() * aty).sum())
    assert abs(lhs - rhs) / abs(lhs) <= TOL


def test_cone_batches_channels_and_accumulate(rng):
    g, geo, plan, torch = _case("cone_circular", B=2, C=3)
    x = rng.random(plan.img_shape).astype(np.float32)
    got = plan.project(torch.from_numpy(x).cuda()).cpu().numpy()
    _, _, one, _ = _case("cone_circular")
    for b in range(2):
        for c in range(3):
            xi = np.ascontiguousarray(x[b:b + 1, ..., c:c + 1])
            np.testing.assert_allclose(got[b:b + 1, ..., c:c + 1], one.project(torch.from_numpy(xi).cuda()).cpu().numpy(),
                                       rtol=1e-6, atol=1e-6)
    y = torch.from_numpy(rng.random(plan.prj_shape).astype(np.float32)).cuda()
    base = torch.full(plan.img_shape, 0.5, device="cuda")
    acc = plan.backproject(y, out=base.clone(), accumulate=True)
    assert torch.allclose(acc, plan.backproject(y) + 0.5, rtol=1e-6, atol=1e-6)


def test_cone_host_api_matches_device(rng):
    from reconnet_b200.reconnet import ReconNet
    g, geo, plan, torch = _case("cone_tomo")
    rn = ReconNet()
    for k in ("nx", "ny", "nz", "dx", "dy", "dz", "cx", "cy", "cz", "nu", "nv", "du", "dv", "off_u", "off_v"):
        setattr(rn, k, getattr(g, k))
    x = rng.random(plan.img_shape).astype(np.float32)
    y = rng.random(plan.prj_shape).astype(np.float32)
    np.testing.assert_array_equal(rn.cSiddonConeProjectionAbitrary4d(x, *geo),
                                  plan.project(torch.from_numpy(x).cuda()).cpu().numpy())
    np.testing.assert_array_equal(rn.cSiddonConeBackprojectionAbitrary4d(y, *geo),
                                  plan.backproject(torch.from_numpy(y).cuda()).cpu().numpy())


def test_cone_ossqs_matches_oracle_loop(rng):
    """cOSSQSConeAbitrary: contiguous subsets (3, 3, 1 views: the corrected
    tail), mask, clamp, lambda."""
    from oracle import oracle as O
    from reconnet_b200.reconnet import ReconNet
    g, geo, plan, torch = _case("cone_tomo")
    dc, du, dv, src = geo
    nview, M_ = dc.shape[0], 3
    truth = (rng.random(plan.img_shape) * 0.5).astype(np.float32)
    prj = O.cone_fp(truth, *geo, g, g.nu, g.nv).astype(np.float32)
    norm = O.cone_bp(O.cone_fp(np.ones_like(truth), *geo, g, g.nu, g.nv).astype(np.float32), *geo, g,
                     (g.nx, g.ny, g.nz)).astype(np.float32)
    mask = (rng.random(truth.shape) > 0.2).astype(np.float32)
    x = np.zeros_like(truth)
    nps = int(np.ceil(nview / M_))
    ref = x.astype(np.float64)
    for k in range(M_):
        sl = slice(k * nps, min(nview, (k + 1) * nps))
        sub = [a[sl] for a in geo]
        r = O.cone_fp(ref.astype(np.float32), *sub, g, g.nu, g.nv) - prj[:, :, sl].astype(np.float64)
        bp = O.cone_bp(r.astype(np.float32), *sub, g, (g.nx, g.ny, g.nz))
        ref = np.clip((ref - 0.8 * M_ * bp / (norm + 1e-6)) * mask, 0.0, 1.0)
    rn = ReconNet()
    for k in ("nx", "ny", "nz", "dx", "dy", "dz", "cx", "cy", "cz", "nu", "nv", "du", "dv", "off_u", "off_v"):
        setattr(rn, k, getattr(g, k))
    got = rn.cSiddonConeAbitraryOSSQS4d(M_, x, prj, norm, *geo, mask=mask, lb=0.0, ub=1.0, lam=0.8)
    assert rel_l2(got, ref) <= 1e-4


def test_cone_rejects_oblique_views():
    from reconnet_b200 import _native as N
    from reconnet_b200.torch_ops import ConeGeometry, ConePlan
    g = ConeGeometry(nx=8, ny=8, nz=8, nu=64, nv=4, du=20.0, dv=1.0)
    src = np.float32([[0, 0, 100]])
    dc = np.float32([[0, 0, -10]])
    du = np.float32([[1, 0, 0]])
    dv = np.float32([[0, 1, 0]])
    with pytest.raises(N.ReconNetError):
        ConePlan(g, dc, du, dv, src)     # edge rays 640 mm sideways over 110 mm: slope > 4


def _sep_case(kind, B=1, C=1):
    """Separable views (detector perpendicular to the main axis, u and v each
    along one lateral axis) beyond the tomosynthesis arc: u along y and v
    along x with more than 32 voxels along v's axis ("swap"); main axis x
    with v along z, the image's contiguous axis ("xmain"); and detector cells
    so fine along u that a voxel's shadow covers more than 32 of them
    ("fine"); and cells so coarse that a block's rays spread over more voxels
    than the forward projector stages in shared memory ("coarse")."""
    import torch
    from reconnet_b200.torch_ops import ConeGeometry, ConePlan
    if kind == "swap":
        g = dict(nx=41, ny=23, nz=5, dx=0.9, dy=1.0, dz=1.3, cx=0.3, cy=0.2, cz=-0.1, nu=30, nv=52, du=1.1,
                 dv=0.95, off_u=-0.2, off_v=0.35)
        n = 4
        a = (np.arange(n) - 1.5) * 0.1
        src = np.stack([np.full(n, 5.0), 300 * np.sin(a), 300 * np.cos(a)], 1)
        dc = np.tile([-0.5, 1.0, -25.0], (n, 1))
        du = np.tile([0.0, 1.0, 0.0], (n, 1))
        dv = np.tile([1.0, 0.0, 0.0], (n, 1))
    elif kind == "xmain":
        g = dict(nx=9, ny=21, nz=37, dx=1.2, dy=0.8, dz=1.0, cx=-0.2, cy=0.4, cz=0.1, nu=28, nv=46, du=0.9,
                 dv=1.0, off_u=0.15, off_v=-0.3)
        n = 3
        a = (np.arange(n) - 1.0) * 0.08
        src = np.stack([350 * np.cos(a), 350 * np.sin(a), np.full(n, 3.0)], 1)
        dc = np.tile([-30.0, 0.5, -0.2], (n, 1))
        du = np.tile([0.0, 1.0, 0.0], (n, 1))
        dv = np.tile([0.0, 0.0, 1.0], (n, 1))
    elif kind == "coarse":
        g = dict(nx=150, ny=61, nz=16, dx=1.0, dy=1.0, dz=1.0, cx=0.3, cy=-0.2, cz=0.0, nu=40, nv=17, du=4.0,
                 dv=3.5, off_u=0.2, off_v=-0.1)
        n = 2
        a = (np.arange(n) - 0.5) * 0.02
        src = np.stack([1000 * np.sin(a), np.full(n, 1.0), 1000 * np.cos(a)], 1)
        dc = np.tile([0.5, 0.0, -20.0], (n, 1))
        du = np.tile([1.0, 0.0, 0.0], (n, 1))
        dv = np.tile([0.0, 1.0, 0.0], (n, 1))
    else:   # fine
        g = dict(nx=6, ny=5, nz=4, dx=1.0, dy=1.0, dz=1.0, cx=0.1, cy=0.0, cz=0.0, nu=330, nv=12, du=0.025,
                 dv=0.6, off_u=0.4, off_v=0.0)
        n = 3
        a = (np.arange(n) - 1.0) * 0.004
        src = np.stack([400 * np.sin(a), np.full(n, 0.3), 400 * np.cos(a)], 1)
        dc = np.tile([0.0, 0.0, -30.0], (n, 1))
        du = np.tile([1.0, 0.0, 0.0], (n, 1))
        dv = np.tile([0.0, 1.0, 0.0], (n, 1))
    geo = tuple(np.ascontiguousarray(v, np.float32) for v in (dc, du, dv, src))
    plan = ConePlan(ConeGeometry(**g), *geo, nbatches=B, nchannels=C)
    return NS(**g), geo, plan, torch


SEP_CASES = ("swap", "xmain", "fine", "coarse")


@pytest.mark.parametrize("kind", SEP_CASES)
def test_cone_separable_matches_oracle(kind, rng):
    from oracle import oracle as O
    g, geo, plan, torch = _sep_case(kind)
    x = rng.random(plan.img_shape).astype(np.float32)
    y = rng.random(plan.prj_shape).astype(np.float32)
    got = plan.project(torch.from_numpy(x).cuda()).cpu().numpy()
    assert rel_l2(got, O.cone_fp(x, *geo, g, g.nu, g.nv)) <= TOL
    got = plan.backproject(torch.from_numpy(y).cuda()).cpu().numpy()
    assert rel_l2(got, O.cone_bp(y, *geo, g, (g.nx, g.ny, g.nz))) <= TOL


@pytest.mark.parametrize("kind", SEP_CASES)
def test_cone_separable_adjoint_and_accumulate(kind, rng):
    g, geo, plan, torch = _sep_case(kind, B=2, C=2)
    x = torch.from_numpy(rng.random(plan.img_shape).astype(np.float32)).cuda()
    y = torch.from_numpy(rng.random(plan.prj_shape).astype(np.float32)).cuda()
    ax = plan.project(x).double()
    aty = plan.backproject(y)
    lhs, rhs = float((ax * y.double()).sum()), float((x.double() * aty.double()).sum())
    assert abs(lhs - rhs) / abs(lhs) <= TOL
    base = torch.full(plan.img_shape, 0.5, device="cuda")
    acc = plan.backproject(y, out=base.clone(), accumulate=True)
    assert torch.allclose(acc, aty + 0.5, rtol=1e-6, atol=1e-6)
