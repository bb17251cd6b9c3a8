"""GPU parity of the sm_100a DD fan kernels against the FP64 oracle, through the
C ABI (device API via FanPlan, host API via the reference-named functions).

Tolerance: relative L2 <= 1e-5 for FP32 projections / backprojections against
the FP64 oracle, and |<Ax,y> - <x,A^T y>| / |<Ax,y>| <= 1e-5 for the matched
pair (FP64 accumulation of the FP32 results)."""
import numpy as np
import pytest

from conftest import rel_l2, small_fan, to_geometry

pytestmark = pytest.mark.gpu

TOL = 1e-5

CASES = {
    "2d": (dict(), 1, 1, 72),
    "offsets": (dict(off_a=0.7, nx=40, ny=52, dx=0.9, dy=1.0), 1, 1, 45),
    "multislice": (dict(nz=3, nv=3), 2, 2, 36),
    "zmix": (dict(nz=3, nv=4, dz=1.5, dv=1.0, off_v=0.3), 1, 2, 30),
    "few_views": (dict(nu=17, da=0.009), 1, 1, 5),
}


def _setup(name, rng):
    import torch
    from reconnet_b200.torch_ops import FanPlan
    kw, B, C, nview = CASES[name]
    g = small_fan(**kw)
    ang = (np.arange(nview) * 2 * np.pi / nview + 0.01 * (name == "few_views")).astype(np.float32)
    plan = FanPlan(to_geometry(g), ang, nbatches=B, nchannels=C)
    x = rng.random((B, g.nx, g.ny, g.nz, C)).astype(np.float32)
    y = rng.random((B, g.nu, nview, g.nv, C)).astype(np.float32)
    return g, ang, plan, x, y, torch


@pytest.mark.parametrize("name", list(CASES))
def test_fp_matches_oracle(name, rng):
    from oracle import oracle as O
    g, ang, plan, x, y, torch = _setup(name, rng)
    got = plan.project(torch.from_numpy(x).cuda()).cpu().numpy()
    plan.check()
    ref = O.fan_fp(x, ang, g, g.nu, g.nv)
    assert rel_l2(got, ref) <= TOL


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("ptype", [0, 1, 2])
def test_bp_matches_oracle(name, ptype, rng):
    from oracle import oracle as O
    g, ang, plan, x, y, torch = _setup(name, rng)
    got = plan.backproject(torch.from_numpy(y).cuda(), ptype).cpu().numpy()
    plan.check()
    ref = O.fan_bp(y, ang, g, (g.nx, g.ny, g.nz), ptype)
    assert rel_l2(got, ref) <= TOL


def test_host_api_matches_device_api(rng):
    from reconnet_b200.reconnet import ReconNet
    g, ang, plan, x, y, torch = _setup("multislice", rng)
    rn = ReconNet()
    for k in ("nx", "ny", "nz", "dx", "dy", "dz", "nu", "nv", "da", "dv", "off_a", "off_v", "dsd", "dso"):
        setattr(rn, k, getattr(g, k))
    fp_h = rn.cDDFanProjection4d(x, ang)
    fp_d = plan.project(torch.from_numpy(x).cuda()).cpu().numpy()
    np.testing.assert_array_equal(fp_h, fp_d)
    for t in (0, 1, 2):
        bp_h = rn.cDDFanBackprojection4d(y, ang, type_projector=t)
        bp_d = plan.backproject(torch.from_numpy(y).cuda(), t).cpu().numpy()
        np.testing.assert_array_equal(bp_h, bp_d)


def test_accumulate_mode(rng):
    g, ang, plan, x, y, torch = _setup("2d", rng)
    yd = torch.from_numpy(y).cuda()
    base = torch.from_numpy(x).cuda()
    ref = base + plan.backproject(yd, 2)
    out = base.clone()
    plan.backproject(yd, 2, out=out, accumulate=True)
    assert torch.allclose(out, ref, rtol=0, atol=0)


def test_ragged_plan_matches_per_slice_plans(rng):
    import torch
    from reconnet_b200.torch_ops import FanPlan
    g = small_fan()
    counts = [31, 47, 20]
    angs = [(np.arange(n) * 2 * np.pi / n).astype(np.float32) for n in counts]
    rag = FanPlan(to_geometry(g), np.concatenate(angs), nbatches=3, nview_per_slice=counts)
    x = rng.random((3, g.nx, g.ny)).astype(np.float32)
    xd = torch.from_numpy(x).cuda()
    p = rag.project(xd)
    y = torch.from_numpy(rng.random(p.shape).astype(np.float32)).cuda()
    b = {t: rag.backproject(y, t) for t in (0, 1, 2)}
    off = 0
    for s, n in enumerate(counts):
        one = FanPlan(to_geometry(g), angs[s])
        ps = one.project(xd[s].reshape(1, g.nx, g.ny, 1, 1).contiguous())
        seg = p[off * g.nu:(off + n) * g.nu].reshape(1, g.nu, n, 1, 1)
        assert torch.equal(ps, seg)
        ys = y[off * g.nu:(off + n) * g.nu].reshape(1, g.nu, n, 1, 1).contiguous()
        for t in (0, 1, 2):
            assert torch.equal(one.backproject(ys, t)[0, :, :, 0, 0], b[t][s])
        off += n


@pytest.mark.parametrize("cfg", ["fan256", "fan512"])
def test_adjoint_full_size(cfg, rng):
    """<Ax, y> = <x, A^T y> at the workload sizes (phantom x, random y)."""
    import torch
    from reconnet_b200 import phantom as P
    from reconnet_b200.torch_ops import FanPlan
    geom = P.geom_fan256() if cfg == "fan256" else P.geom_fan512()
    nview = 720 if cfg == "fan256" else 864
    plan = FanPlan(geom, P.uniform_angles(nview))
    x = P.ellipse_phantom(geom.nx, geom.ny, geom.dx, geom.dy, rng)[None, :, :, None, None]
    xd = torch.from_numpy(x).cuda()
    Ax = plan.project(xd)
    yd = torch.rand_like(Ax)
    Aty = plan.backproject(yd, 2)
    plan.check()
    lhs = float((Ax.double() * yd.double()).sum())
    rhs = float((xd.double() * Aty.double()).sum())
    assert abs(lhs - rhs) / abs(lhs) <= TOL


def test_fan256_full_size_fp_bp_vs_oracle(rng):
    import torch
    from oracle import oracle as O
    from reconnet_b200 import phantom as P
    from reconnet_b200.torch_ops import FanPlan
    geom = P.geom_fan256()
    ang = P.uniform_angles(720)
    plan = FanPlan(geom, ang)
    x = P.ellipse_phantom(geom.nx, geom.ny, geom.dx, geom.dy, rng)[None, :, :, None, None]
    got = plan.project(torch.from_numpy(x).cuda()).cpu().numpy()
    ref = O.fan_fp(x, ang, geom, geom.nu, 1)
    assert rel_l2(got, ref) <= TOL
    y = ref.astype(np.float32)
    for t in (0, 2):
        bp = plan.backproject(torch.from_numpy(y).cuda(), t).cpu().numpy()
        assert rel_l2(bp, O.fan_bp(y, ang, geom, (geom.nx, geom.ny, 1), t)) <= TOL


def test_fan512_slice_fp_vs_oracle(rng):
    """One full 512x512, 888-channel slice (the batched workload's slice)."""
    import torch
    from oracle import oracle as O
    from reconnet_b200 import phantom as P
    from reconnet_b200.torch_ops import FanPlan
    geom = P.geom_fan512()
    ang = P.uniform_angles(600)[::4].copy()
    plan = FanPlan(geom, ang)
    x = P.ellipse_phantom(geom.nx, geom.ny, geom.dx, geom.dy, rng)[None, :, :, None, None]
    got = plan.project(torch.from_numpy(x).cuda()).cpu().numpy()
    ref = O.fan_fp(x, ang, geom, geom.nu, 1)
    assert rel_l2(got, ref) <= TOL
    y = ref.astype(np.float32)
    bp = plan.backproject(torch.from_numpy(y).cuda(), 2).cpu().numpy()
    assert rel_l2(bp, O.fan_bp(y, ang, geom, (geom.nx, geom.ny, 1), 2)) <= TOL


@pytest.mark.parametrize("tf", [0, 1, 2, 3])
def test_filter_matches_oracle(tf, rng):
    import torch
    from oracle import oracle as O
    from reconnet_b200.torch_ops import filter_sino
    g = small_fan(nu=97, da=0.003, off_a=0.4)
    s = rng.random((2, g.nu, 50, 2, 1)).astype(np.float32)
    got = filter_sino(torch.from_numpy(s).cuda(), to_geometry(g), tf).cpu().numpy()
    assert rel_l2(got, O.filter_sino(s, g, tf)) <= TOL
    got_p = filter_sino(torch.from_numpy(s).cuda(), to_geometry(g), tf, fan=False).cpu().numpy()
    assert rel_l2(got_p, O.filter_sino(s, g, tf, fan=False)) <= TOL


# Channel counts whose transform lengths N = 2^logN >= 2nu - 1 cover every
# residue of logN mod 3 (the FFT fuses radix-2 levels three at a time, so the
# remainder picks the radix-4 / radix-2 passes and which pass carries the
# spectrum product) and the largest lengths (N = 8192 and 16384, one signal
# per CTA).  Odd view counts leave the last CTA partly filled.
@pytest.mark.parametrize("nu", [40, 150, 300, 1500, 3000, 5000, 8000])
def test_filter_fft_lengths_match_oracle(nu, rng):
    import torch
    from oracle import oracle as O
    from reconnet_b200.torch_ops import filter_sino
    g = small_fan(nu=nu, da=0.9 / nu, off_a=0.3)
    nview = 7 if nu >= 3000 else 13
    s = rng.random((1, nu, nview, 1, 1)).astype(np.float32)
    for tf in (0, 2):
        got = filter_sino(torch.from_numpy(s).cuda(), to_geometry(g), tf).cpu().numpy()
        assert rel_l2(got, O.filter_sino(s, g, tf)) <= TOL, (nu, tf)


@pytest.mark.parametrize("nu", [150, 300, 736, 888])
def test_filter_kernel_forms_agree(nu, rng):
    """The register four-step FFT (transform lengths 512-2048), the
    shared-memory FFT and the direct product give the same filtered
    sinograms; with short-scan weights too."""
    import torch
    from reconnet_b200 import _native as N
    from reconnet_b200.torch_ops import FanGeometry, filter_sino, shortscan_weights
    geom = FanGeometry(nu=nu, da=0.9 / nu, off_a=0.25)
    s = torch.from_numpy(rng.random((2, nu, 67, 1, 1)).astype(np.float32)).cuda()
    outs = []
    try:
        for form in (0, 1, 2):
            N.check(N.lib.rn_filter_set_form(form))
            outs.append(filter_sino(s, geom, 2).cpu().numpy())
    finally:
        N.lib.rn_filter_set_form(0)
    assert rel_l2(outs[0], outs[2]) <= 2e-6 and rel_l2(outs[1], outs[2]) <= 2e-6


def test_filter_more_planes_than_grid_rows(rng):
    """More (batch, row, channel) planes than one grid dimension holds
    (65,535): the kernels loop over the planes."""
    import torch
    from oracle import oracle as O
    from reconnet_b200.torch_ops import filter_sino
    g = small_fan(nu=16, da=0.01, nv=65600)
    s = rng.random((1, 16, 3, 65600, 1)).astype(np.float32)
    got = filter_sino(torch.from_numpy(s).cuda(), to_geometry(g), 0).cpu().numpy()
    ref = O.filter_sino(s, g, 0)
    assert rel_l2(got, ref) <= TOL
    assert rel_l2(got[..., -100:, :], ref[..., -100:, :]) <= TOL     # the planes past the first grid pass


def test_filter_host_api_full_size(rng):
    from oracle import oracle as O
    from reconnet_b200 import phantom as P
    from reconnet_b200.reconnet import ReconNet
    rn = ReconNet()
    rn.nu, rn.da = 736, 1.2858 / 1085.6
    s = rng.random((1, 736, 720, 1)).astype(np.float32)
    got = rn.cFilter3d(s, 2)
    ref = O.filter_sino(s[..., None, :], P.geom_fan256(), 2)[..., 0, :]
    assert rel_l2(got, ref) <= TOL


def test_tv_matches_oracle(rng):
    import torch
    from oracle import oracle as O
    from reconnet_b200.reconnet import ReconNet
    from reconnet_b200.torch_ops import tv_sqs
    img = rng.random((3, 33, 41)).astype(np.float32) * 0.02
    grad, norm, tv = tv_sqs(torch.from_numpy(img).cuda())
    for s in range(3):
        g2, n2, t2 = O.tv_sqs(img[s])
        assert rel_l2(grad[s].cpu().numpy(), g2) <= TOL
        assert rel_l2(norm[s].cpu().numpy(), n2) <= TOL
        assert abs(float(tv[s]) - t2) / t2 <= TOL
    gh, nh, th = ReconNet().cTVSQS2d(img[0][None, :, :, None])
    g2, n2, t2 = O.tv_sqs(img[0])
    assert rel_l2(gh[0, :, :, 0], g2) <= TOL and abs(th - t2) / t2 <= TOL


@pytest.mark.parametrize("beta,ptype", [(0.0, 2), (0.02, 2), (0.0, 0), (0.02, 3)])
def test_sqs_update_matches_oracle(beta, ptype, rng):
    """rn_fan_sqs_update: DD forward with backprojector 0 / 2, or the Siddon pair (3)."""
    import torch
    from oracle import oracle as O
    from reconnet_b200.torch_ops import FanPlan
    g = small_fan()
    nview, M = 48, 4
    ang = (np.arange(nview) * 2 * np.pi / nview).astype(np.float32)
    x = (rng.random((g.nx, g.ny)) * 0.02).astype(np.float32)
    truth = (rng.random((g.nx, g.ny)) * 0.02).astype(np.float32)
    sino = O.fan_fp(truth[None, :, :, None, None], ang, g, g.nu, 1)[0, :, :, 0, 0].astype(np.float32)
    w = (0.5 + rng.random(sino.shape)).astype(np.float32)
    norm = O.fan_bp((O.fan_fp(np.ones((1, g.nx, g.ny, 1, 1), np.float32), ang, g, g.nu, 1)[0, :, :, 0, 0] * w)
                    .astype(np.float32)[None, :, :, None, None], ang, g, (g.nx, g.ny, 1), min(ptype, 2))[0, :, :, 0, 0]
    norm = norm.astype(np.float32)
    views = np.arange(1, nview, M)
    ref = O.sqs_subset_update(x, sino, w, norm, ang, views, g, M, lam=0.9, beta=beta, lb=0.0, ub=1.0,
                              bp_type=min(ptype, 2), projector="siddon" if ptype == 3 else "dd")
    sp = FanPlan(to_geometry(g), ang[views])
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()
    xo = torch.empty((1, g.nx, g.ny, 1, 1), device="cuda")
    sp.sqs_update(xo, dev(x[None, :, :, None, None]), dev(sino[:, views][None, :, :, None, None]),
                  dev(w[:, views][None, :, :, None, None]), dev(norm[None, :, :, None, None]), lam=0.9, beta=beta,
                  n_subsets=M, lb=0.0, ub=1.0, type_projector=ptype)
    assert rel_l2(xo.cpu().numpy()[0, :, :, 0, 0], ref) <= TOL


@pytest.mark.parametrize("projector", ["siddon", "dd"])
def test_cossqs_host_matches_oracle_loop(projector, rng):
    """cOSSQS (ossqs.cu:12: the Siddon pair) and cDDFanOSSQS (the DD pair,
    matched backprojector) with contiguous subsets and the corrected tail."""
    from oracle import oracle as O
    from reconnet_b200.reconnet import ReconNet
    g = small_fan()
    nview, M = 50, 4            # 50 = 13+13+13+11: the tail subset has 11 views
    ang = (np.arange(nview) * 2 * np.pi / nview).astype(np.float32)
    truth = (rng.random((g.nx, g.ny)) * 0.02).astype(np.float32)
    sino = O.fan_fp(truth[None, :, :, None, None], ang, g, g.nu, 1)[0, :, :, 0, 0].astype(np.float32)
    w = np.ones_like(sino)
    norm = O.fan_bp(O.fan_fp(np.ones((1, g.nx, g.ny, 1, 1), np.float32), ang, g, g.nu, 1).astype(np.float32), ang, g,
                    (g.nx, g.ny, 1), 2)[0, :, :, 0, 0].astype(np.float32)
    x = np.zeros((g.nx, g.ny), np.float32)
    nps = int(np.ceil(nview / M))
    ref = x.astype(np.float64)
    for k in range(M):
        views = np.arange(k * nps, min(nview, (k + 1) * nps))
        ref = O.sqs_subset_update(ref.astype(np.float32), sino, w, norm, ang, views, g, M, bp_type=2,
                                  projector=projector)
    rn = ReconNet()
    for k in ("nx", "ny", "nz", "dx", "dy", "dz", "nu", "nv", "da", "dv", "off_a", "off_v", "dsd", "dso"):
        setattr(rn, k, getattr(g, k))
    fn = rn.cSiddonFanOSSQS3d if projector == "siddon" else rn.cDDFanOSSQS3d
    got = fn(M, x[None, :, :, None], sino[None, :, :, None], norm[None, :, :, None], w[None, :, :, None], ang,
             type_projector=2)[0, :, :, 0]
    assert rel_l2(got, ref) <= 1e-4   # four chained steps


def test_tomo_matches_oracle(rng):
    from oracle import oracle as O
    from reconnet_b200.reconnet import ReconNet
    from test_oracle_cpu import _tomo_setup
    g, dc, src = _tomo_setup(rng)
    rn = ReconNet()
    rn.nx, rn.ny, rn.nz, rn.nu, rn.nv = 16, 14, 6, 24, 20
    for k in ("dx", "dy", "dz", "cx", "cy", "cz", "du", "dv", "off_u", "off_v"):
        setattr(rn, k, getattr(g, k))
    img = rng.random((2, 16, 14, 6, 1)).astype(np.float32)
    got = rn.cDDTomoProjection4d(img, dc, src)
    assert rel_l2(got, O.tomo_fp(img, dc, src, g, 24, 20)) <= TOL
    prj = rng.random(got.shape).astype(np.float32)
    gb = rn.cDDTomoBackprojection4d(prj, dc, src)
    assert rel_l2(gb, O.tomo_bp(prj, dc, src, g, (16, 14, 6), 0)) <= TOL
    # device API, both pre-weight modes
    import ctypes
    import torch
    from reconnet_b200 import _native as N
    fpb, bpb = ctypes.c_size_t(), ctypes.c_size_t()
    N.lib.rn_tomo_sat_bytes(16, 14, 6, 24, 5, 20, ctypes.byref(fpb), ctypes.byref(bpb))
    sat = torch.empty(max(fpb.value, bpb.value) // 8 + 1, dtype=torch.float64, device="cuda")
    dprj = torch.from_numpy(prj).cuda()
    ddc, dsrc = torch.from_numpy(dc).cuda(), torch.from_numpy(src).cuda()
    for mode in (0, 1):
        out = torch.empty((2, 16, 14, 6, 1), device="cuda")
        N.check(N.lib.rn_tomo_backproject(out.data_ptr(), dprj.data_ptr(), ddc.data_ptr(), dsrc.data_ptr(),
                                          sat.data_ptr(), 2, 1, 16, 14, 6, g.dx, g.dy, g.dz, g.cx, g.cy, g.cz, 24,
                                          5, 20, g.du, g.dv, g.off_u, g.off_v, mode,
                                          torch.cuda.current_stream().cuda_stream))
        assert rel_l2(out.cpu().numpy(), O.tomo_bp(prj, dc, src, g, (16, 14, 6), mode)) <= TOL


def test_tomo_negative_magnification_matches_oracle(rng):
    """A detector beyond the source (magnification r < 0): the voxels' detector
    faces then run against y, and the backprojection sweeps its rows in the
    reverse order; ny = 21 leaves a warp with 5 of its 8 voxel rows."""
    from oracle import oracle as O
    from reconnet_b200.reconnet import ReconNet
    from test_oracle_cpu import _tomo_setup
    g, dc, src = _tomo_setup(rng)
    dc[:, 2] = 700.0
    rn = ReconNet()
    rn.nx, rn.ny, rn.nz, rn.nu, rn.nv = 16, 21, 6, 24, 20
    for k in ("dx", "dy", "dz", "cx", "cy", "cz", "du", "dv", "off_u", "off_v"):
        setattr(rn, k, getattr(g, k))
    img = rng.random((1, 16, 21, 6, 1)).astype(np.float32)
    got = rn.cDDTomoProjection4d(img, dc, src)
    assert rel_l2(got, O.tomo_fp(img, dc, src, g, 24, 20)) <= TOL
    prj = rng.random(got.shape).astype(np.float32)
    gb = rn.cDDTomoBackprojection4d(prj, dc, src)
    assert rel_l2(gb, O.tomo_bp(prj, dc, src, g, (16, 21, 6), 0)) <= TOL


def test_invalid_arguments_raise():
    import torch
    from reconnet_b200 import _native as N
    from reconnet_b200.torch_ops import FanPlan
    g = small_fan()
    plan = FanPlan(to_geometry(g), np.zeros(4, np.float32))
    y = torch.zeros(plan.sino_shape, device="cuda")
    with pytest.raises(N.ReconNetError):
        plan.backproject(y, 7)
    with pytest.raises(ValueError):
        plan.project(torch.zeros((1, 3, 3, 1, 1), device="cuda"))
    with pytest.raises(N.ReconNetError):   # source inside the image
        FanPlan(to_geometry(small_fan(dso=20.0, dsd=40.0)), np.zeros(4, np.float32))


def test_streamed_pair_matches_single_plan(rng):
    """StreamedFanPair (slice groups, overlapped host copies) returns exactly
    what one ragged plan computes, call after call."""
    import torch
    from reconnet_b200.torch_ops import FanPlan, StreamedFanPair
    g = small_fan()
    counts = np.array([40, 52, 33, 45, 37], np.int64)
    angles = np.concatenate([(np.arange(n) * 2 * np.pi / n + 0.1 * s).astype(np.float32)
                             for s, n in enumerate(counts)])
    geom = to_geometry(g)
    plan = FanPlan(geom, angles, nbatches=len(counts), nview_per_slice=counts)
    pair = StreamedFanPair(geom, angles, counts, groups=3)
    assert pair.updates() == plan.fp_updates() + plan.bp_updates()
    out = torch.empty((len(counts), g.nx, g.ny), dtype=torch.float32).pin_memory()
    for call in range(3):
        imgs = torch.from_numpy(rng.random((len(counts), g.nx, g.ny)).astype(np.float32)).pin_memory()
        pair(imgs, out).synchronize()
        pair.check()
        ref = plan.backproject(plan.project(imgs.cuda()), 2).cpu()
        assert torch.equal(out, ref), call


@pytest.mark.parametrize("op", ["project", "backproject"])
def test_device_wait_timeout_is_reported_and_recoverable(op, rng):
    """A spin limit of zero polls makes every chunk wait of the kernels give
    up at once: the kernels record RN_ERR_TIMEOUT, wait (bounded) for their
    own bulk copies in flight and return, with no fault.  check() reports it;
    with the default limit the same plan then computes the right result."""
    import torch
    from oracle import oracle as O
    from reconnet_b200 import _native as N
    from reconnet_b200.torch_ops import FanPlan
    g = small_fan()
    ang = (np.arange(40) * 2 * np.pi / 40).astype(np.float32)
    plan = FanPlan(to_geometry(g), ang)
    x = rng.random((1, g.nx, g.ny, 1, 1)).astype(np.float32)
    y = rng.random((1, g.nu, ang.size, 1, 1)).astype(np.float32)
    run = (lambda: plan.project(torch.from_numpy(x).cuda())) if op == "project" else \
        (lambda: plan.backproject(torch.from_numpy(y).cuda(), 2))
    plan.set_spin_limit(0)
    run()
    with pytest.raises(N.ReconNetError) as e:
        plan.check()
    assert e.value.code == N.RN_ERR_TIMEOUT
    plan.set_spin_limit(-1)
    got = run().cpu().numpy()
    plan.check()
    ref = O.fan_fp(x, ang, g, g.nu, 1) if op == "project" else O.fan_bp(y, ang, g, (g.nx, g.ny, 1), 2)
    assert rel_l2(got, ref) <= TOL
