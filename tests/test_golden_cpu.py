"""The oracle against golden vectors produced by the reference's own CUDA
kernels (tests/golden/make_golden.py, run on a B200 with the reference
library built from its sources).

The reference reads its prefix sums through linear-filtering textures, so the
oracle is compared twice:
  * with exact weights (the oracle proper): bounded by the texture error;
  * with the B200 texture unit's weights as measured (oracle mode 3: 8-bit
    fractions after the coordinate clamp, exact depth marginals, round-half-
    down splits in the other dimensions; pinned to hardware fetches by
    tests/golden/ref_texfetch.npz).  What then remains is the reference's
    __sinf/__cosf: a replica of its forward kernel with accurate sinf/cosf
    and hardware textures differs from it by 3.8e-4 (fan2d) and 1.0e-3
    (fan256) on X-class views, and the residuals below sit at those figures.
The X-class views carry ten times the Y-class texture error because their
rows are blended 50/50 in the texture's height dimension, which the unit
splits unevenly when the depth weight is odd.
Tomosynthesis, filter and TV paths use no textures and agree to ~1e-6."""
import glob
import os
from types import SimpleNamespace as NS

import numpy as np
import pytest

from conftest import ROOT, rel_l2
from oracle import oracle as O

GOLDEN = os.path.join(ROOT, "tests", "golden")
FAN = sorted(glob.glob(os.path.join(GOLDEN, "ref_fan*.npz")))


def _fan(path):
    d = dict(np.load(path))
    g = NS(**{k: float(d[k]) for k in ("dx", "dy", "dz", "da", "dv", "off_a", "off_v", "dsd", "dso")})
    dims = {k: int(d[k]) for k in ("nx", "ny", "nz", "nu", "nv")}
    return d, g, dims


@pytest.fixture(autouse=True)
def _restore_quant():
    yield
    O.set_tex_quant(0)


def test_golden_files_present():
    assert len(FAN) >= 4
    assert os.path.exists(os.path.join(GOLDEN, "ref_tv.npz"))
    assert os.path.exists(os.path.join(GOLDEN, "ref_tomo.npz"))


@pytest.mark.parametrize("path", FAN, ids=[os.path.basename(p)[4:-4] for p in FAN])
def test_fan_fp_vs_reference(path):
    d, g, n = _fan(path)
    fp = O.fan_fp(d["img"], d["angles"], g, n["nu"], n["nv"])
    assert rel_l2(fp, d["fp"]) < 4e-3
    xv = np.array([O.view_is_x(a) for a in d["angles"]])
    # with the measured texture weights only the reference's __sinf/__cosf remain
    O.set_tex_quant(3)
    emu = O.fan_fp(d["img"], d["angles"], g, n["nu"], n["nv"])
    x_bound = 1.2e-3 if "fan256" in path else 6e-4      # fan256: its trig floor is 1.02e-3
    assert rel_l2(emu[:, :, xv], d["fp"][:, :, xv]) < x_bound
    if (~xv).any():
        assert rel_l2(emu[:, :, ~xv], d["fp"][:, :, ~xv]) < 1.5e-4


@pytest.mark.parametrize("path", FAN, ids=[os.path.basename(p)[4:-4] for p in FAN])
@pytest.mark.parametrize("ptype", [0, 1])
def test_fan_bp_vs_reference(path, ptype):
    d, g, n = _fan(path)
    shape = (n["nx"], n["ny"], n["nz"])
    exact = O.fan_bp(d["sino_in"], d["angles"], g, shape, ptype)
    assert rel_l2(exact, d[f"bp{ptype}"]) < 1e-3
    O.set_tex_quant(1)     # texture emulation: weights rounded to 1/256
    emu = O.fan_bp(d["sino_in"], d["angles"], g, shape, ptype)
    assert rel_l2(emu, d[f"bp{ptype}"]) < 1.2e-4
    O.set_tex_quant(3)     # the measured weights (the backprojection fetches vary one coordinate)
    assert rel_l2(O.fan_bp(d["sino_in"], d["angles"], g, shape, ptype), d[f"bp{ptype}"]) < 1.2e-4
    # rounding fits the hardware better than truncation
    O.set_tex_quant(2)
    trunc = O.fan_bp(d["sino_in"], d["angles"], g, shape, ptype)
    assert rel_l2(trunc, d[f"bp{ptype}"]) > rel_l2(emu, d[f"bp{ptype}"])


@pytest.mark.parametrize("path", FAN, ids=[os.path.basename(p)[4:-4] for p in FAN])
def test_filter_vs_reference(path):
    d, g, n = _fan(path)
    for tf in (0, 2):
        if f"filt{tf}" in d:
            assert rel_l2(O.filter_sino(d["sino_in"], g, tf), d[f"filt{tf}"]) < 2e-6


def test_tv_vs_reference():
    d = dict(np.load(os.path.join(GOLDEN, "ref_tv.npz")))
    grad, norm, tv = O.tv_sqs(d["img"][0, :, :, 0])
    assert rel_l2(grad, d["grad"][0, :, :, 0]) < 1e-6
    assert rel_l2(norm, d["norm"][0, :, :, 0]) < 1e-6
    assert abs(tv - d["tv"]) / tv < 1e-5     # the reference sums in FP32


def test_tomo_vs_reference():
    d = dict(np.load(os.path.join(GOLDEN, "ref_tomo.npz")))
    g = NS(**{k: float(d[k]) for k in ("dx", "dy", "dz", "cx", "cy", "cz", "du", "dv", "off_u", "off_v")})
    nu, nv = int(d["nu"]), int(d["nv"])
    assert rel_l2(O.tomo_fp(d["img"], d["det_center"], d["src"], g, nu, nv), d["fp"]) < 1e-5
    shape = d["img"].shape[1:4]
    assert rel_l2(O.tomo_bp(d["prj_in"], d["det_center"], d["src"], g, shape, 0), d["bp"]) < 1e-5
    # the reference's BP weights only view 0 (one-row pre-weight grid); the
    # all-views variant differs by far more than the tolerance
    assert rel_l2(O.tomo_bp(d["prj_in"], d["det_center"], d["src"], g, shape, 1), d["bp"]) > 0.1


SIDDON = sorted(glob.glob(os.path.join(GOLDEN, "ref_siddon*.npz")))


@pytest.mark.parametrize("path", SIDDON, ids=[os.path.basename(p)[4:-4] for p in SIDDON])
def test_siddon_vs_reference(path):
    """Exact FP64 crossings against the reference's incremental FP32 tracing
    with __sinf/__cosf ray directions (Siddon.cu:240-375); its backprojector
    accumulates with float atomics."""
    d, g, n = _fan(path)
    fp = O.siddon_fp(d["img"], d["angles"], g, n["nu"], n["nv"])
    assert rel_l2(fp, d["fp"]) < 1e-4      # measured 3.9e-5 / 4.3e-5
    bp = O.siddon_bp(d["sino_in"], d["angles"], g, (n["nx"], n["ny"], n["nz"]))
    assert rel_l2(bp, d["bp"]) < 2e-4      # measured 6.6e-5 / 1.1e-4


OSSQS = os.path.join(GOLDEN, "ref_ossqs_siddon.npz")


def ossqs_oracle_loop(d, g):
    """The oracle's OS-SQS pass with contiguous subsets and the Siddon pair,
    on a cOSSQS golden case (tests/golden/make_golden.py ossqs_case)."""
    M = int(d["n_subsets"])
    nview = d["angles"].size
    nps = nview // M
    x = d["x0"][0, :, :, 0, 0]
    sino, w, norm = d["sino"][0, :, :, 0, 0], d["w"][0, :, :, 0, 0], d["norm"][0, :, :, 0, 0]
    for k in range(M):
        x = O.sqs_subset_update(x.astype(np.float32), sino, w, norm, d["angles"], np.arange(k * nps, (k + 1) * nps),
                                g, M, lam=float(d["lam"]), lb=float(d["lb"]), ub=float(d["ub"]), projector="siddon")
    return x


def test_ossqs_siddon_vs_reference():
    """The oracle's OS-SQS loop against the reference's cOSSQS
    (ossqs.cu:12-161: Siddon pair, Minus2D / Multiply2D / Divide2D /
    ValueCrop2D) on the same inputs."""
    d, g, _ = _fan(OSSQS)
    assert rel_l2(ossqs_oracle_loop(d, g), d["res"][0, :, :, 0, 0]) < 1e-4   # measured 2.8e-5


PIXEL = sorted(glob.glob(os.path.join(GOLDEN, "ref_pixel*.npz")))


@pytest.mark.parametrize("path", PIXEL, ids=[os.path.basename(p)[4:-4] for p in PIXEL])
def test_pixel_bp_vs_reference(path):
    """The pixel-driven backprojection (PixelDriven.cu:11-62) reads its
    sinogram through a linear-filtering texture with 8-bit weights and uses
    __sinf/__cosf; the oracle is checked with exact weights and with the
    weights rounded to 1/256."""
    d, g, n = _fan(path)
    exact = O.pixel_bp(d["sino_in"], d["angles"], g, (n["nx"], n["ny"], n["nz"]))
    O.set_tex_quant(1)
    rounded = O.pixel_bp(d["sino_in"], d["angles"], g, (n["nx"], n["ny"], n["nz"]))
    print(f"{os.path.basename(path)}: exact {rel_l2(exact, d['bp']):.3g}, rounded {rel_l2(rounded, d['bp']):.3g}")
    assert rel_l2(exact, d["bp"]) < 2e-3      # measured 1.1e-4 / 9.7e-4
    assert rel_l2(rounded, d["bp"]) < 5e-4    # measured 8.6e-6 / 2.3e-4


TVISO = sorted(glob.glob(os.path.join(GOLDEN, "ref_tviso*.npz")))


@pytest.mark.parametrize("path", TVISO, ids=[os.path.basename(p)[4:-4] for p in TVISO])
def test_tv_iso_vs_reference(path):
    """The prior solver's isotropic TV surrogate (PriorFunctionSolver/TVSQS.cu),
    FP32 in the reference, against the FP64 restatement."""
    d = dict(np.load(path))
    s1, s2, var = O.tv_iso_sqs(d["img"], int(d["ndim"]), float(d["eps"]))
    assert rel_l2(var, d["var"]) < 1e-6     # measured 3.5e-8 / 3.6e-8
    assert rel_l2(s2, d["s2"]) < 1e-6      # measured 1.7e-8 / 1.9e-8
    assert rel_l2(s1, d["s1"]) < 1e-6      # measured 4.7e-8 / 4.8e-8


CONE = sorted(glob.glob(os.path.join(GOLDEN, "ref_cone*.npz")))


@pytest.mark.parametrize("path", CONE, ids=[os.path.basename(p)[4:-4] for p in CONE])
def test_cone_vs_reference(path):
    """Exact FP64 crossings against the reference's incremental FP32 Siddon
    (SiddonCone.cu:20-67; its backprojector accumulates with float atomics)."""
    d = dict(np.load(path))
    g = NS(**{k: float(d[k]) for k in ("dx", "dy", "dz", "cx", "cy", "cz", "du", "dv", "off_u", "off_v")})
    n = {k: int(d[k]) for k in ("nx", "ny", "nz", "nu", "nv")}
    geo = [d[k] for k in ("det_center", "det_u", "det_v", "src")]
    fp = O.cone_fp(d["img"], *geo, g, n["nu"], n["nv"])
    bp = O.cone_bp(d["prj_in"], *geo, g, (n["nx"], n["ny"], n["nz"]))
    assert rel_l2(fp, d["fp"]) < 1e-5      # measured 1.1e-6 - 1.3e-6
    assert rel_l2(bp, d["bp"]) < 1e-5      # measured 1.8e-6 - 2.7e-6


SHORTSCAN = os.path.join(GOLDEN, "ref_shortscan.npz")


@pytest.mark.parametrize("case", ["c736", "c736_off", "c96", "c200_wide"])
def test_shortscan_weights_vs_reference(case):
    """The oracle's Parker / Riess weights against the reference's own
    ParkerWeighting / RiessWeighting run on the same angles
    (tests/golden/make_shortscan_golden.py); the fixtures are float32, so the
    bound is their rounding."""
    d = np.load(SHORTSCAN)
    nu, da, off = d[f"{case}_geom"]
    ang = d[f"{case}_angles"]
    nu = int(nu)
    assert np.abs(O.shortscan_weights(ang, nu, da, off, "parker") - d[f"{case}_parker"]).max() < 1.2e-7
    riess = O.shortscan_weights(ang, nu, da, off, "riess")
    assert np.abs(riess - d[f"{case}_riess"]).max() < 1.2e-7
    assert np.abs(O.shortscan_weights(ang, nu, da, off, "riess", 12, 0.1) - d[f"{case}_riess_s12"]).max() < 1.2e-7
    # the reference keeps only channel 0 of the middle views unsmoothed; the
    # whole-view reading of the method gives different weights
    whole = O.shortscan_weights(ang, nu, da, off, "riess", mask_all=True)
    assert np.abs(whole - d[f"{case}_riess"]).max() > 0.1


TEXFETCH = os.path.join(GOLDEN, "ref_texfetch.npz")


@pytest.mark.skipif(not os.path.exists(TEXFETCH), reason="texture-fetch golden vectors not generated")
def test_texture_model_vs_hardware_fetches():
    """The oracle's texture model (mode 3) against fetches made by the B200's
    texture unit (tests/golden/texfetch.cu): the fan2d prefix tables with the
    reference's layouts and addressing at X- and Y-class coordinates across
    and beyond the image, and an impulse texture at pairs of fractional
    coordinates.  Equal to FP32 rounding."""
    d = np.load(TEXFETCH)
    mx = O.tex_fetch(d["px"][:, :, None], (0, 0, 1), d["cx"])
    assert np.max(np.abs(mx - d["vx"]) / np.maximum(np.abs(d["vx"]), 1e-3)) < 2e-7
    my = O.tex_fetch(d["py"][:, :, None], (0, 1, 0), d["cy"])
    assert np.max(np.abs(my - d["vy"]) / np.maximum(np.abs(d["vy"]), 1e-3)) < 2e-7
    imp = np.zeros((8, 8, 1), np.float32)
    imp[4, 4, 0] = 1.0
    mi = O.tex_fetch(imp, (0, 0, 1), d["ci"])
    assert np.array_equal(mi.astype(np.float32), d["vi"])
    # the same fetches with each dimension's weight rounded alone miss by up to 1/256
    assert np.abs(O.tex_fetch(imp, (0, 0, 1), d["ci"], quant=1) - d["vi"]).max() > 1e-3
