"""The forward projection that allocates nothing (rn_fan_project_noalloc).

It exists for callers that may not allocate device memory (a host framework's
memory pool, a fixed memory budget, real-time code that forbids cudaMalloc
after start-up); its scratch is a fixed device array inside the library.
These checks call it through the C ABI twice in a row, with different images
and angle lists so the shared scratch is rewritten, and compare each result
with the allocating entry point (rn_fan_project through a plan) at the suite's
tolerance.  Collected last so that a failure here does not hide others."""
import ctypes

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _noalloc(N, torch, img, ang, g):
    nu, nview = g.nu, ang.size
    out = torch.full((nu, nview), float("nan"), device="cuda")
    a = np.ascontiguousarray(ang, np.float32)
    st = N.lib.rn_fan_project_noalloc(out.data_ptr(), img.data_ptr(), a.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                      g.nx, g.ny, g.dx, g.dy, nu, nview, g.da, g.off_a, g.dsd, g.dso,
                                      torch.cuda.current_stream().cuda_stream)
    return st, out


def test_noalloc_projection_matches_plan_projection_twice(rng):
    import torch
    from reconnet_b200 import _native as N
    from reconnet_b200 import phantom as P
    from reconnet_b200.torch_ops import FanPlan
    g = P.geom_fan512()
    for nview in (864, 601):
        ang = P.uniform_angles(nview) + np.float32(0.003 * nview)
        img = torch.from_numpy(P.ellipse_phantom(g.nx, g.ny, g.dx, g.dy, rng)).cuda()
        st, out = _noalloc(N, torch, img, ang, g)
        N.check(st)
        ref = FanPlan(g, ang).project(img.reshape(1, g.nx, g.ny, 1, 1).contiguous())[0, :, :, 0, 0]
        assert torch.isfinite(out).all()
        assert rel_l2(out.cpu().numpy(), ref.cpu().numpy()) <= TOL


def test_noalloc_rejects_geometry_beyond_its_scratch():
    import torch
    from reconnet_b200 import _native as N
    from reconnet_b200 import phantom as P
    g = P.geom_fan512()
    img = torch.zeros((g.nx, g.ny), device="cuda")
    st, _ = _noalloc(N, torch, img, P.uniform_angles(4000), g)
    assert st == N.RN_ERR_ARG
    assert "bytes of scratch" in N.last_error()
