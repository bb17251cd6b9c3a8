"""Siddon fan projector pair on the GPU against the FP64 oracle (exact
crossings; oracle pinned to the reference's Siddon kernels by the golden
vectors), its adjoint, the reference-named host entry points, and the
reference's own Siddon kernels run live.

Tolerance: relative L2 <= 1e-5 against the FP64 oracle, |<Ax,y> - <x,A^T y>| /
|<Ax,y>| <= 1e-5."""
import numpy as np
import pytest

from conftest import rel_l2, small_fan, to_geometry

pytestmark = pytest.mark.gpu

TOL = 1e-5

CASES = {
    "2d": (dict(), 1, 1, 72, 0.0),
    "offsets": (dict(off_a=0.7, nx=40, ny=52, dx=0.9, dy=1.0), 1, 1, 45, 0.0),
    # views at multiples of 90 degrees: rays parallel to the grid lines
    "axis_views": (dict(), 1, 1, 8, None),
    "multislice": (dict(nz=3, nv=3, off_v=0.25), 2, 2, 36, 0.01),
    "few_views": (dict(nu=17, da=0.009), 1, 1, 5, 0.01),
}


def _setup(name, rng):
    import torch
    from reconnet_b200.torch_ops import FanPlan
    kw, B, C, nview, shift = CASES[name]
    g = small_fan(**kw)
    if shift is None:
        ang = (np.arange(nview) * np.pi / 4).astype(np.float32)
    else:
        ang = (np.arange(nview) * 2 * np.pi / nview + shift).astype(np.float32)
    plan = FanPlan(to_geometry(g), ang, nbatches=B, nchannels=C)
    x = rng.random((B, g.nx, g.ny, g.nz, C)).astype(np.float32)
    y = rng.random((B, g.nu, nview, g.nv, C)).astype(np.float32)
    return g, ang, plan, x, y, torch


@pytest.mark.parametrize("name", list(CASES))
def test_siddon_fp_matches_oracle(name, rng):
    from oracle import oracle as O
    g, ang, plan, x, y, torch = _setup(name, rng)
    got = plan.project(torch.from_numpy(x).cuda(), siddon=True).cpu().numpy()
    plan.check()
    assert rel_l2(got, O.siddon_fp(x, ang, g, g.nu, g.nv)) <= TOL


@pytest.mark.parametrize("name", list(CASES))
def test_siddon_bp_matches_oracle(name, rng):
    from oracle import oracle as O
    from reconnet_b200 import _native as N
    g, ang, plan, x, y, torch = _setup(name, rng)
    got = plan.backproject(torch.from_numpy(y).cuda(), N.RN_TYPE_SIDDON).cpu().numpy()
    plan.check()
    assert rel_l2(got, O.siddon_bp(y, ang, g, (g.nx, g.ny, g.nz))) <= TOL


@pytest.mark.parametrize("name", ["2d", "multislice", "axis_views"])
def test_siddon_adjoint(name, rng):
    from reconnet_b200 import _native as N
    g, ang, plan, x, y, torch = _setup(name, rng)
    ax = plan.project(torch.from_numpy(x).cuda(), siddon=True).double()
    aty = plan.backproject(torch.from_numpy(y).cuda(), N.RN_TYPE_SIDDON).double()
    lhs = float((ax * torch.from_numpy(y).cuda().double()).sum())
    rhs = float((torch.from_numpy(x).cuda().double() * aty).sum())
    assert abs(lhs - rhs) / abs(lhs) <= TOL


def test_siddon_host_api_matches_device(rng):
    from reconnet_b200 import _native as N
    from reconnet_b200.reconnet import ReconNet
    g, ang, plan, x, y, torch = _setup("multislice", rng)
    rn = ReconNet()
    for k in ("nx", "ny", "nz", "dx", "dy", "dz", "nu", "nv", "da", "dv", "off_a", "off_v", "dsd", "dso"):
        setattr(rn, k, getattr(g, k))
    np.testing.assert_array_equal(rn.cSiddonFanProjection4d(x, ang),
                                  plan.project(torch.from_numpy(x).cuda(), siddon=True).cpu().numpy())
    np.testing.assert_array_equal(rn.cSiddonFanBackprojection4d(y, ang),
                                  plan.backproject(torch.from_numpy(y).cuda(), N.RN_TYPE_SIDDON).cpu().numpy())


def test_siddon_full_size_slice(rng):
    """A slice of the 64-slice batch workload (512 x 512 at 0.7 mm, 888 channels) with 96 views."""
    import torch
    from oracle import oracle as O
    from reconnet_b200 import _native as N
    from reconnet_b200 import phantom as P
    from reconnet_b200.torch_ops import FanPlan
    g = P.geom_fan512()
    ang = P.uniform_angles(96)
    img = P.ellipse_phantom(g.nx, g.ny, g.dx, g.dy, rng)[None, :, :, None, None]
    plan = FanPlan(g, ang)
    fp = plan.project(torch.from_numpy(img).cuda(), siddon=True)
    assert rel_l2(fp.cpu().numpy(), O.siddon_fp(img, ang, g, g.nu, 1)) <= TOL
    bp = plan.backproject(fp, N.RN_TYPE_SIDDON).cpu().numpy()
    assert rel_l2(bp, O.siddon_bp(fp.cpu().numpy(), ang, g, (g.nx, g.ny, 1))) <= TOL
    plan.check()


def test_cossqs_matches_oracle_on_reference_case():
    """cOSSQS on the committed cOSSQS golden case (inputs from the reference's
    own Siddon kernels) against the oracle's OS-SQS loop with the Siddon pair."""
    import os
    from conftest import ROOT
    from test_golden_cpu import _fan, ossqs_oracle_loop
    from reconnet_b200.reconnet import ReconNet
    d, g, n = _fan(os.path.join(ROOT, "tests", "golden", "ref_ossqs_siddon.npz"))
    rn = ReconNet()
    for k in ("dx", "dy", "dz", "da", "dv", "off_a", "off_v", "dsd", "dso"):
        setattr(rn, k, getattr(g, k))
    for k, v in n.items():
        setattr(rn, k, v)
    got = rn.cSiddonFanOSSQS4d(int(d["n_subsets"]), d["x0"], d["sino"], d["norm"], d["w"], d["angles"],
                               lb=float(d["lb"]), ub=float(d["ub"]), lam=float(d["lam"]))
    assert rel_l2(got[0, :, :, 0, 0], ossqs_oracle_loop(d, g)) <= 1e-4   # four chained steps
