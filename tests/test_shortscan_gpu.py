"""Short-scan weights on the GPU (csrc/shortscan.cu, rn_fan_shortscan_weights)
against the reference's own ParkerWeighting / RiessWeighting
(tests/golden/ref_shortscan.npz) and the FP64 oracle; and the FBP chain with
the weights fused into the ramp filter's load (rn_filter_weighted).

Tolerances: the weights are FP32 outputs of FP64 arithmetic, so 2.5e-7
absolute against the float32 fixtures (two float32 roundings); the FBP chain
1e-5 relative L2 against the oracle's chain."""
import os

import numpy as np
import pytest

from conftest import ROOT, rel_l2, small_fan, to_geometry

pytestmark = pytest.mark.gpu

GOLDEN = np.load(os.path.join(ROOT, "tests", "golden", "ref_shortscan.npz"))
CASES = ["c736", "c736_off", "c96", "c200_wide"]


def _case(case):
    nu, da, off = GOLDEN[f"{case}_geom"]
    return int(nu), float(da), float(off), GOLDEN[f"{case}_angles"]


@pytest.mark.parametrize("case", CASES)
def test_device_weights_match_reference(case):
    import torch
    from reconnet_b200.torch_ops import FanGeometry, shortscan_weights
    nu, da, off, ang = _case(case)
    g = FanGeometry(nu=nu, da=da, off_a=off)
    a = torch.from_numpy(ang).cuda()
    assert np.abs(shortscan_weights(a, g, "parker").cpu().numpy() - GOLDEN[f"{case}_parker"]).max() <= 2.5e-7
    assert np.abs(shortscan_weights(a, g, "riess").cpu().numpy() - GOLDEN[f"{case}_riess"]).max() <= 2.5e-7
    got = shortscan_weights(a, g, "riess", sigma=12, theta=0.1).cpu().numpy()
    assert np.abs(got - GOLDEN[f"{case}_riess_s12"]).max() <= 2.5e-7


@pytest.mark.parametrize("case", CASES)
def test_whole_view_exception_matches_oracle(case):
    import torch
    from oracle import oracle as O
    from reconnet_b200.torch_ops import FanGeometry, shortscan_weights
    nu, da, off, ang = _case(case)
    got = shortscan_weights(torch.from_numpy(ang).cuda(), FanGeometry(nu=nu, da=da, off_a=off), "riess",
                            whole_view_exception=True).cpu().numpy()
    assert np.abs(got - O.shortscan_weights(ang, nu, da, off, "riess", mask_all=True)).max() <= 2.5e-7


def test_reference_named_functions_match_device():
    import torch
    from reconnet_b200.reconnet import ParkerWeighting, ReconNet, RiessWeighting
    from reconnet_b200.torch_ops import FanGeometry, shortscan_weights
    nu, da, off, ang = _case("c96")
    rn = ReconNet()
    rn.nu, rn.da, rn.off_a, rn.angles = nu, da, off, ang
    g = FanGeometry(nu=nu, da=da, off_a=off)
    a = torch.from_numpy(ang).cuda()
    pw = ParkerWeighting(rn)
    assert pw.shape == (1, nu, ang.size, 1)
    assert np.array_equal(pw[0, :, :, 0], shortscan_weights(a, g, "parker").cpu().numpy())
    assert np.array_equal(RiessWeighting(rn)[0, :, :, 0], shortscan_weights(a, g, "riess").cpu().numpy())


def test_bad_kind_is_an_error():
    import torch
    from reconnet_b200 import _native as N
    w = torch.empty(16, 8, device="cuda")
    a = torch.zeros(8, device="cuda")
    st = N.lib.rn_fan_shortscan_weights(w.data_ptr(), a.data_ptr(), 16, 8, 0.01, 0.0, 7, 30.0, 0.1, 0,
                                        torch.cuda.current_stream().cuda_stream)
    assert st == N.RN_ERR_ARG


@pytest.mark.parametrize("kind", ["parker", "riess"])
def test_fbp_with_fused_weights_matches_oracle_chain(kind, rng):
    """fbp(weights=...) multiplies the weights inside the filter's load; the
    oracle chain multiplies first, filters, then backprojects pixel-driven."""
    import torch
    from oracle import oracle as O
    from reconnet_b200.torch_ops import FanPlan, fbp, shortscan_weights
    g = small_fan(nx=64, ny=64, dx=1.0, dy=1.0, nu=96, da=0.0022, off_a=0.3)
    geom = to_geometry(g)
    nview = 121
    ang = (np.arange(nview) * (np.pi + g.nu * g.da + 0.05) / (nview - 1)).astype(np.float32)
    w = shortscan_weights(torch.from_numpy(ang).cuda(), geom, kind)
    y = rng.random((2, g.nu, nview, 1, 1)).astype(np.float32)
    plan = FanPlan(geom, ang, nbatches=2)
    got = fbp(torch.from_numpy(y).cuda(), plan, geom, 2, w).cpu().numpy()
    wo = O.shortscan_weights(ang, g.nu, g.da, g.off_a, kind).astype(np.float32)[None, :, :, None, None]
    filt = O.filter_sino((y * wo).astype(np.float32), g, 2, True).astype(np.float32)
    assert rel_l2(got, O.pixel_bp(filt, ang, g, (g.nx, g.ny, 1))) <= 1e-5
