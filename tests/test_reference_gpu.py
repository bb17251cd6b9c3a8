"""The reference's own CUDA kernels (oracle/_ref, compiled from the
reference sources) against this library on the same GPU and inputs.

The reference fetches its prefix sums through linear-filtering textures whose
interpolation weights have 8 fractional bits, and uses __sinf/__cosf, so it
differs from exact arithmetic by ~1e-3 (relative L2); that is the bound used
here.  The tight parity bar (1e-5) is against the FP64 oracle in
test_fan_gpu.py; the oracle itself is pinned to these reference outputs by
tests/test_golden_cpu.py."""
import os
import time

import numpy as np
import pytest

from conftest import ROOT, rel_l2

pytestmark = pytest.mark.gpu

REF = os.path.join(ROOT, "oracle", "_ref", "libreconnet_ref.so")
REF_TOL = 5e-3


@pytest.fixture(scope="module")
def ref():
    if not os.path.exists(REF):
        pytest.skip("reference library not built (make -C oracle ref needs the reference sources)")
    import sys
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import make_golden
    return make_golden


@pytest.mark.parametrize("name", ["fan2d", "fan_offsets", "fan_multislice", "fan256"])
def test_fan_vs_reference_kernels(ref, name, rng):
    from reconnet_b200.reconnet import ReconNet
    lib = ref.load_ref()
    out = ref.fan_case(lib, name, rng)
    rn = ReconNet()
    for k in ("nx", "ny", "nz", "dx", "dy", "dz", "nu", "nv", "da", "dv", "off_a", "off_v", "dsd", "dso"):
        setattr(rn, k, out[k].item() if k not in ("nx", "ny", "nz", "nu", "nv") else int(out[k]))
    fp = rn.cDDFanProjection4d(out["img"], out["angles"])
    assert rel_l2(fp, out["fp"]) <= REF_TOL
    # the definition, with the texture unit's measured weights, against the
    # live reference: only its __sinf/__cosf remain (fan256's floor 1.0e-3)
    from oracle import oracle as O
    from types import SimpleNamespace
    g = SimpleNamespace(**{k: float(out[k]) for k in ("dx", "dy", "dz", "da", "dv", "off_a", "off_v", "dsd", "dso")})
    O.set_tex_quant(3)
    try:
        emu = O.fan_fp(out["img"], out["angles"], g, int(out["nu"]), int(out["nv"]))
    finally:
        O.set_tex_quant(0)
    assert rel_l2(emu, out["fp"]) <= (1.2e-3 if name == "fan256" else 6e-4)
    for t in (0, 1):
        bp = rn.cDDFanBackprojection4d(out["sino_in"], out["angles"], type_projector=t)
        assert rel_l2(bp, out[f"bp{t}"]) <= REF_TOL
    for tf in (0, 2):
        if f"filt{tf}" in out:
            assert rel_l2(rn.cFilter4d(out["sino_in"], tf), out[f"filt{tf}"]) <= 1e-4


def test_tv_and_tomo_vs_reference_kernels(ref, rng):
    from reconnet_b200.reconnet import ReconNet
    lib = ref.load_ref()
    tv = ref.tv_case(lib, rng)
    g, n, t = ReconNet().cTVSQS2d(tv["img"])
    assert rel_l2(g, tv["grad"]) <= 1e-6 and rel_l2(n, tv["norm"]) <= 1e-6
    assert abs(t - tv["tv"]) / tv["tv"] <= 1e-5
    to = ref.tomo_case(lib, rng)
    rn = ReconNet()
    rn.nx, rn.ny, rn.nz = to["img"].shape[1:4]
    rn.nu, rn.nv = int(to["nu"]), int(to["nv"])
    for k in ("dx", "dy", "dz", "cx", "cy", "cz", "du", "dv", "off_u", "off_v"):
        setattr(rn, k, to[k].item())
    assert rel_l2(rn.cDDTomoProjection4d(to["img"], to["det_center"], to["src"]), to["fp"]) <= 1e-5
    assert rel_l2(rn.cDDTomoBackprojection4d(to["prj_in"], to["det_center"], to["src"]), to["bp"]) <= 1e-5


def test_reference_host_call_timing(ref, rng):
    """Times the reference's and this library's host entry points (the
    reference's published path: ctypes FP + BP incl. allocation and copies)
    on the default 512x512 / 736 x 720 geometry and prints both."""
    import ctypes
    from reconnet_b200.reconnet import ReconNet
    lib = ref.load_ref()
    rn = ReconNet()
    img = np.zeros((1, 512, 512, 1, 1), np.float32)
    img[0, 128:384, 128:384] = 0.02
    ang = np.array(rn.angles, np.float32)
    sino = np.zeros((1, rn.nu, ang.size, 1, 1), np.float32)
    bp = np.zeros_like(img)
    p = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    args = (1, 1, 512, 512, 1, 1.0, 1.0, 2.0, rn.nu, ang.size, 1, rn.da, rn.dv, 0.0, 0.0, rn.dsd, rn.dso)
    ts = {}
    calls = [("reference", lambda: (lib.cDistanceDrivenFanProjection(p(sino), p(img), p(ang), *args, 0),
                                    lib.cDistanceDrivenFanBackprojection(p(bp), p(sino), p(ang), *args, 0))),
             ("b200", lambda: (rn.cDDFanProjection4d(img, ang), rn.cDDFanBackprojection4d(sino, ang)))]
    if hasattr(lib, "cSiddonFanProjection"):
        # the Siddon pair, the other path with a published host-call time
        calls += [("reference_siddon", lambda: (lib.cSiddonFanProjection(p(sino), p(img), p(ang), *args, 0),
                                                lib.cSiddonFanBackprojection(p(bp), p(sino), p(ang), *args, 0))),
                  ("b200_siddon", lambda: (rn.cSiddonFanProjection4d(img, ang),
                                           rn.cSiddonFanBackprojection4d(sino, ang)))]
    for name, fn in calls:
        fn()
        t0 = time.perf_counter()
        for _ in range(5):
            fn()
        ts[name] = (time.perf_counter() - t0) / 5
    print(f"\nFP+BP host call, 512x512 736x720: reference {ts['reference']*1e3:.2f} ms, "
          f"b200 {ts['b200']*1e3:.2f} ms")
    assert ts["b200"] < ts["reference"]
    if "b200_siddon" in ts:
        print(f"Siddon FP+BP host call: reference {ts['reference_siddon']*1e3:.2f} ms, "
              f"b200 {ts['b200_siddon']*1e3:.2f} ms")
        assert ts["b200_siddon"] < ts["reference_siddon"]


def test_siddon_vs_reference_kernels(ref, rng):
    """The reference's Siddon kernels (incremental FP32 tracing, __sinf/__cosf
    ray directions, float atomics in the backprojector) against the Siddon
    pair here: measured ~4e-5 (FP) / ~1e-4 (BP) apart."""
    from reconnet_b200.reconnet import ReconNet
    lib = ref.load_ref()
    if not hasattr(lib, "cSiddonFanProjection"):
        pytest.skip("reference library built without Siddon.cu")
    for name, out in ref.siddon_case(lib, rng).items():
        rn = ReconNet()
        for k in ("nx", "ny", "nz", "dx", "dy", "dz", "nu", "nv", "da", "dv", "off_a", "off_v", "dsd", "dso"):
            setattr(rn, k, out[k].item() if k not in ("nx", "ny", "nz", "nu", "nv") else int(out[k]))
        assert rel_l2(rn.cSiddonFanProjection4d(out["img"], out["angles"]), out["fp"]) <= 2e-4, name
        assert rel_l2(rn.cSiddonFanBackprojection4d(out["sino_in"], out["angles"]), out["bp"]) <= 4e-4, name


def test_cossqs_vs_reference(ref, rng):
    """cOSSQS here (Siddon pair, like ossqs.cu:81) against the reference's
    cOSSQS on the same inputs, nview a multiple of nviewPerSubset."""
    from reconnet_b200.reconnet import ReconNet
    lib = ref.load_ref()
    if not hasattr(lib, "cOSSQS"):
        pytest.skip("reference library built without ossqs.cu")
    d = ref.ossqs_case(lib, rng)
    rn = ReconNet()
    for k in ("nx", "ny", "nz", "dx", "dy", "dz", "nu", "nv", "da", "dv", "off_a", "off_v", "dsd", "dso"):
        setattr(rn, k, d[k].item() if k not in ("nx", "ny", "nz", "nu", "nv") else int(d[k]))
    got = rn.cSiddonFanOSSQS4d(int(d["n_subsets"]), d["x0"], d["sino"], d["norm"], d["w"], d["angles"],
                               lb=float(d["lb"]), ub=float(d["ub"]), lam=float(d["lam"]))
    err = rel_l2(got, d["res"])
    print(f"cOSSQS vs reference: {err:.3g}")
    assert err <= 1e-4   # measured 2.8e-5


def test_pixel_bp_vs_reference_kernels(ref, rng):
    """The reference's bpFanKernel3D (texture reads with 8-bit weights) against
    the pixel-driven backprojection here."""
    from reconnet_b200.reconnet import ReconNet
    lib = ref.load_ref()
    if not hasattr(lib, "cPixelDrivenFanBackprojection"):
        pytest.skip("reference library built without PixelDriven.cu")
    for name, out in ref.pixel_case(lib, rng).items():
        rn = ReconNet()
        for k in ("nx", "ny", "nz", "dx", "dy", "dz", "nu", "nv", "da", "dv", "off_a", "off_v", "dsd", "dso"):
            setattr(rn, k, out[k].item() if k not in ("nx", "ny", "nz", "nu", "nv") else int(out[k]))
        err = rel_l2(rn.cPixelBackprojection4d(out["sino_in"], out["angles"]), out["bp"])
        print(f"pixel-driven BP vs reference ({name}): {err:.3g}")
        assert err <= REF_TOL, name


def test_cone_vs_reference_kernels(ref, rng):
    """The reference's Siddon cone kernels (SiddonCone.cu) and its cone
    OS-SQS (ossqs.cu:163-333) against this library on the same inputs."""
    from reconnet_b200.reconnet import ReconNet
    lib = ref.load_ref()
    if not hasattr(lib, "cSiddonConeProjectionAbitrary"):
        pytest.skip("reference library built without SiddonCone.cu")
    for name, d in ref.cone_case(lib, rng).items():
        rn = ReconNet()
        for k in ("nx", "ny", "nz", "nu", "nv"):
            setattr(rn, k, int(d[k]))
        for k in ("dx", "dy", "dz", "cx", "cy", "cz", "du", "dv", "off_u", "off_v"):
            setattr(rn, k, d[k].item())
        geo = [d[k] for k in ("det_center", "det_u", "det_v", "src")]
        efp = rel_l2(rn.cSiddonConeProjectionAbitrary4d(d["img"], *geo), d["fp"])
        ebp = rel_l2(rn.cSiddonConeBackprojectionAbitrary4d(d["prj_in"], *geo), d["bp"])
        print(f"{name}: fp {efp:.3g} bp {ebp:.3g}")
        assert efp <= 1e-5 and ebp <= 1e-5, name      # measured ~1e-6 / ~3e-6
        if "ossqs_res" in d:
            nview = d["det_center"].shape[0]
            got = rn.cSiddonConeAbitraryOSSQS4d(nview, d["ossqs_x0"], d["fp"], d["ossqs_norm"], *geo,
                                                mask=d["ossqs_mask"], lb=0.0, ub=1.0, lam=float(d["ossqs_lam"]))
            eos = rel_l2(got, d["ossqs_res"])
            print(f"{name}: cone OS-SQS {eos:.3g}")
            assert eos <= 1e-4      # measured 7e-6
