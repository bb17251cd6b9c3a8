"""GPU parity of the cylindrical-detector cone-beam DD pair (csrc/cyl.cu)
against the FP64 oracle (oracle.cpp, cyl_view_terms), through the C ABI.

This geometry has no reference kernel (the reference's DistanceDriven3D.cu is
a flat-detector tomosynthesis pair), so parity rests on the oracle and on the
adjoint identity.  Tolerances: relative L2 <= 1e-5 for the FP32 projections
and backprojections against the FP64 oracle; |<Ax,y> - <x,A^T y>| / |<Ax,y>|
<= 1e-5 with the dot products taken in FP64."""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _geom(**kw):
    from reconnet_b200.torch_ops import CylGeometry
    base = dict(nx=40, ny=36, nz=12, dx=1.0, dy=1.0, dz=1.0, nu=64, nv=8, da=0.0025, dv=2.0, dsd=1085.6, dso=595.0)
    base.update(kw)
    return CylGeometry(**base)


CASES = {
    "basic": dict(),
    "anisotropic_offsets": dict(dx=0.9, dy=1.1, dz=0.7, cx=3.0, cy=-2.0, cz=1.5, off_a=0.7, off_v=-0.4),
    "many_rows": dict(nv=70, dv=0.5),                        # three row groups, the last one ragged
    "tall_detector": dict(nz=8, nv=24, dv=3.0),               # row edges above and below the volume
    "wide_fan": dict(nu=40, da=0.02, nz=6, nv=5),             # edge rays far from the central ray
}


def _angles(n, start=0.0):
    return (start + np.arange(n) * 2 * np.pi / n).astype(np.float32)


@pytest.mark.parametrize("name", list(CASES))
def test_cyl_pair_matches_oracle(name, rng):
    import torch
    from oracle import oracle as O
    from reconnet_b200.torch_ops import CylPlan
    g = _geom(**CASES[name])
    ang = _angles(45, 0.013)
    plan = CylPlan(g, ang, nbatches=2)
    x = rng.random(plan.vol_shape).astype(np.float32)
    y = rng.random(plan.prj_shape).astype(np.float32)
    ax = plan.project(torch.from_numpy(x).cuda())
    aty = plan.backproject(torch.from_numpy(y).cuda())
    assert rel_l2(ax.cpu().numpy(), O.cyl_fp(x, ang, g)) <= TOL
    assert rel_l2(aty.cpu().numpy(), O.cyl_bp(y, ang, g, (g.nx, g.ny, g.nz))) <= TOL
    lhs = float((ax.double() * torch.from_numpy(y).cuda().double()).sum())
    rhs = float((torch.from_numpy(x).cuda().double() * aty.double()).sum())
    assert abs(lhs - rhs) / abs(lhs) <= TOL
    assert plan.launches() == 4          # FP: z prefix table + FP; BP: row tables + BP


def test_cyl_views_on_class_boundaries(rng):
    """Views at multiples of 45 degrees (the X/Y class switch and the axes)."""
    import torch
    from oracle import oracle as O
    from reconnet_b200.torch_ops import CylPlan
    g = _geom()
    ang = (np.arange(16) * np.pi / 8).astype(np.float32)
    plan = CylPlan(g, ang)
    x = rng.random(plan.vol_shape).astype(np.float32)
    y = rng.random(plan.prj_shape).astype(np.float32)
    assert rel_l2(plan.project(torch.from_numpy(x).cuda()).cpu().numpy(), O.cyl_fp(x, ang, g)) <= TOL
    assert rel_l2(plan.backproject(torch.from_numpy(y).cuda()).cpu().numpy(),
                  O.cyl_bp(y, ang, g, (g.nx, g.ny, g.nz))) <= TOL


def test_cyl_uniform_volume_central_ray():
    """A uniform volume's central ray at view 0 runs along y through all ny
    voxel rows: ny dy times the value."""
    import torch
    from reconnet_b200.torch_ops import CylPlan
    g = _geom(nu=65, nv=9)
    plan = CylPlan(g, np.zeros(1, np.float32))
    p = plan.project(torch.full(plan.vol_shape, 0.02, device="cuda")).cpu().numpy()
    assert p[0, 32, 0, 4] == pytest.approx(0.02 * g.ny * g.dy, rel=1e-6)


def test_cyl_rejects_source_inside_volume():
    from reconnet_b200 import _native as N
    from reconnet_b200.torch_ops import CylPlan
    with pytest.raises(N.ReconNetError):
        CylPlan(_geom(dso=20.0, dsd=40.0), _angles(4))


def test_cyl_full_size(rng):
    """The cone-beam workload at full size: 512 x 512 x 128 voxels of
    0.8 x 0.8 x 1.0 mm, 736 x 64 cells, 984 views over 360 degrees.  The
    adjoint identity over all views on the GPU, and parity with the oracle on
    four of the views (the oracle's cost grows with the views)."""
    import torch
    from oracle import oracle as O
    from reconnet_b200.phantom import ellipsoid_phantom
    from reconnet_b200.torch_ops import CylGeometry, CylPlan
    g = CylGeometry()
    ang = _angles(984)
    plan = CylPlan(g, ang)
    x = ellipsoid_phantom(g.nx, g.ny, g.nz, g.dx, g.dy, g.dz, np.random.default_rng(5), device="cuda")[None].contiguous()
    y = torch.rand(plan.prj_shape, device="cuda")
    ax = plan.project(x)
    aty = plan.backproject(y)
    lhs = float((ax.double() * y.double()).sum())
    rhs = float((x.double() * aty.double()).sum())
    assert abs(lhs - rhs) / abs(lhs) <= TOL
    sel = np.array([0, 123, 370, 801])
    sub = CylPlan(g, ang[sel])
    xs = x.cpu().numpy()
    got = sub.project(x).cpu().numpy()
    assert np.array_equal(got, ax[:, :, sel, :].cpu().numpy())       # a view's projection depends on it alone
    assert rel_l2(got, O.cyl_fp(xs, ang[sel], g)) <= TOL
    ys = np.ascontiguousarray(y[:, :, sel, :].cpu().numpy())
    assert rel_l2(sub.backproject(torch.from_numpy(ys).cuda()).cpu().numpy(),
                  O.cyl_bp(ys, ang[sel], g, (g.nx, g.ny, g.nz))) <= TOL
