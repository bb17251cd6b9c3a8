"""Pixel-driven FBP backprojection (PixelDriven.cu:11-141) on the GPU against
the FP64 oracle, the reference-named host entry point against the device
plan, and the device FBP chain (short-scan weights, ramp filter, pixel-driven
backprojection).

Tolerance: relative L2 <= 1e-5 against the FP64 oracle."""
import numpy as np
import pytest

from conftest import rel_l2, small_fan, to_geometry

pytestmark = pytest.mark.gpu

TOL = 1e-5

CASES = {
    "2d": (dict(), 1, 1, 72, 0.0),
    "offsets": (dict(off_a=0.7, nx=40, ny=52, dx=0.9, dy=1.0), 1, 1, 45, 0.3),
    "axis_views": (dict(), 1, 1, 8, None),
    # slices between detector rows, rows beyond the volume, channels, batches
    "multislice": (dict(nz=3, nv=4, dz=1.3, off_v=0.35), 2, 2, 36, 0.01),
    "few_views": (dict(nu=17, da=0.009), 1, 1, 5, 0.01),
    # the detector narrower than the image: pixels beyond the edge cells
    "narrow_detector": (dict(nu=24), 1, 1, 20, 0.1),
}


def _setup(name, rng):
    from reconnet_b200.torch_ops import FanPlan
    kw, B, C, nview, shift = CASES[name]
    g = small_fan(**kw)
    if shift is None:
        ang = (np.arange(nview) * np.pi / 4).astype(np.float32)
    else:
        ang = (np.arange(nview) * 2 * np.pi / nview + shift).astype(np.float32)
    plan = FanPlan(to_geometry(g), ang, nbatches=B, nchannels=C)
    y = rng.random((B, g.nu, nview, g.nv, C)).astype(np.float32)
    return g, ang, plan, y


@pytest.mark.parametrize("name", list(CASES))
def test_pixel_bp_matches_oracle(name, rng):
    import torch
    from oracle import oracle as O
    from reconnet_b200 import _native as N
    g, ang, plan, y = _setup(name, rng)
    got = plan.backproject(torch.from_numpy(y).cuda(), N.RN_TYPE_PIXEL).cpu().numpy()
    plan.check()
    assert rel_l2(got, O.pixel_bp(y, ang, g, (g.nx, g.ny, g.nz))) <= TOL


def test_pixel_bp_accumulates(rng):
    import torch
    from reconnet_b200 import _native as N
    g, ang, plan, y = _setup("2d", rng)
    dy = torch.from_numpy(y).cuda()
    base = torch.full(plan.img_shape, 0.25, device="cuda")
    one = plan.backproject(dy, N.RN_TYPE_PIXEL)
    acc = plan.backproject(dy, N.RN_TYPE_PIXEL, out=base.clone(), accumulate=True)
    assert torch.allclose(acc, one + 0.25, rtol=1e-6, atol=1e-6)


def test_pixel_host_api_matches_device(rng):
    import torch
    from reconnet_b200 import _native as N
    from reconnet_b200.reconnet import ReconNet
    g, ang, plan, y = _setup("multislice", rng)
    rn = ReconNet()
    for k in ("nx", "ny", "nz", "dx", "dy", "dz", "nu", "nv", "da", "dv", "off_a", "off_v", "dsd", "dso"):
        setattr(rn, k, getattr(g, k))
    np.testing.assert_array_equal(rn.cPixelBackprojection4d(y, ang),
                                  plan.backproject(torch.from_numpy(y).cuda(), N.RN_TYPE_PIXEL).cpu().numpy())
    y3 = y[:1, :, :, :1, :]
    rn.nz, rn.nv = 1, 1
    got = rn.cPixelBackprojection3d(y3[..., 0, :], ang)
    assert got.shape == (1, g.nx, g.ny, 2)


def test_pixel_full_size_slice(rng):
    """512 x 512 at 0.7 mm, 888 channels, 720 views: the bench geometry."""
    import torch
    from oracle import oracle as O
    from reconnet_b200 import _native as N
    from reconnet_b200.phantom import geom_fan512
    from reconnet_b200.torch_ops import FanPlan
    geom = geom_fan512()
    ang = (np.arange(720) * 2 * np.pi / 720).astype(np.float32)
    y = rng.random((1, geom.nu, 720, 1, 1)).astype(np.float32)
    plan = FanPlan(geom, ang)
    got = plan.backproject(torch.from_numpy(y).cuda(), N.RN_TYPE_PIXEL).cpu().numpy()
    assert rel_l2(got, O.pixel_bp(y, ang, geom, (geom.nx, geom.ny, 1))) <= TOL


def test_fbp_chain_matches_oracle_and_reconstructs(rng):
    """fbp = Parker weights x ramp filter x pixel-driven backprojection against
    the same chain in the oracle, on a short scan; and a full-scan FBP of a DD
    projection reproduces the phantom."""
    import torch
    from oracle import oracle as O
    from reconnet_b200.phantom import ellipse_phantom
    from reconnet_b200.reconnet import ParkerWeighting, ReconNet
    from reconnet_b200.torch_ops import FanPlan, fbp
    g = small_fan(nx=64, ny=64, dx=1.0, dy=1.0, nu=96, da=0.0022)
    geom = to_geometry(g)
    # short scan: pi + fan angle, Parker weights
    fan = g.nu * g.da
    nview = 120
    ang = (np.arange(nview) * (np.pi + fan) / (nview - 1)).astype(np.float32)
    rn = ReconNet()
    for k in ("nu", "da", "off_a"):
        setattr(rn, k, getattr(g, k))
    rn.angles = ang
    w = ParkerWeighting(rn).astype(np.float32)[..., None]            # [1, nu, nview, 1, 1]
    y = rng.random((1, g.nu, nview, 1, 1)).astype(np.float32)
    plan = FanPlan(geom, ang)
    got = fbp(torch.from_numpy(y).cuda(), plan, geom, 0, torch.from_numpy(w).cuda()).cpu().numpy()
    filt = O.filter_sino((y * w).astype(np.float32), g, 0, True).astype(np.float32)
    assert rel_l2(got, O.pixel_bp(filt, ang, g, (g.nx, g.ny, 1))) <= 1e-5
    # full scan FBP of a phantom
    ang = (np.arange(360) * 2 * np.pi / 360).astype(np.float32)
    plan = FanPlan(geom, ang)
    img = ellipse_phantom(g.nx, g.ny, g.dx, g.dy, np.random.default_rng(3))[None, :, :, None, None]
    img = np.ascontiguousarray(img, np.float32)
    prj = plan.project(torch.from_numpy(img).cuda())
    rec = fbp(prj, plan, geom).cpu().numpy()
    inner = np.s_[:, 8:-8, 8:-8]
    assert rel_l2(rec[inner], img[inner]) < 0.15
