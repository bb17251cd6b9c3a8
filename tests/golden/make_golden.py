"""Generate golden vectors from the reference's own CUDA kernels.

Runs on a GPU machine: loads ``oracle/_ref/libreconnet_ref.so`` (the
reference's ReconNet4D_no_tf sources compiled by ``make -C oracle ref``) and
calls its C entry points through ctypes exactly as python/ReconNet_no_tf.py
does, on small seeded inputs.  Writes ``tests/golden/ref_*.npz`` (inputs,
geometry and reference outputs); the CPU test suite checks the oracle against
these files.

    python tests/golden/make_golden.py [outdir]
    python tests/golden/make_golden.py --siddon [outdir]   (the Siddon pair only)
    python tests/golden/make_golden.py --ossqs [outdir]    (cOSSQS only)
    python tests/golden/make_golden.py --pixel [outdir]    (pixel-driven backprojection only)
    python tests/golden/make_golden.py --prior [outdir]    (the prior solver's TV, oracle/_ref/libprior_ref.so)
    python tests/golden/make_golden.py --cone [outdir]     (the Siddon cone pair and cone OS-SQS)
"""
import ctypes
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.path.join(ROOT, "oracle", "_ref", "libreconnet_ref.so")

_f = ctypes.c_float
_i = ctypes.c_int
_fp = ctypes.POINTER(ctypes.c_float)


def load_ref(path=REF):
    lib = ctypes.CDLL(path)
    fan = [_fp, _fp, _fp] + [_i, _i, _i, _i, _i, _f, _f, _f, _i, _i, _i, _f, _f, _f, _f, _f, _f, _i]
    lib.cDistanceDrivenFanProjection.argtypes = fan
    lib.cDistanceDrivenFanBackprojection.argtypes = fan
    filt = [_fp, _fp, _i, _i, _i, _i, _i, _f, _f, _f, _f, _f, _f, _i, _i]
    lib.cFilterFanFilter.argtypes = filt
    lib.cFilterParallelFilter.argtypes = filt
    lib.cTVSQS2D.argtypes = [_fp, _fp, _fp, _i, _i]
    lib.cTVSQS2D.restype = _f
    tomo = [_fp, _fp, _fp, _fp] + [_i, _i, _i, _i, _i, _f, _f, _f, _f, _f, _f, _i, _i, _i, _f, _f, _f, _f]
    lib.cDistanceDrivenTomoProjection.argtypes = tomo
    lib.cDistanceDrivenTomoBackprojection.argtypes = tomo
    if hasattr(lib, "cSiddonFanProjection"):
        lib.cSiddonFanProjection.argtypes = fan
        lib.cSiddonFanBackprojection.argtypes = fan
    if hasattr(lib, "cPixelDrivenFanBackprojection"):
        lib.cPixelDrivenFanBackprojection.argtypes = fan
    if hasattr(lib, "cSiddonConeProjectionAbitrary"):
        lib.cSiddonConeProjectionAbitrary.argtypes = [_fp] * 6 + tomo[4:]
        lib.cSiddonConeBackprojectionAbitrary.argtypes = [_fp] * 6 + tomo[4:]
    if hasattr(lib, "cOSSQSConeAbitrary"):
        lib.cOSSQSConeAbitrary.argtypes = [_fp] * 9 + [_f, _f, _i, _i] + tomo[4:] + [_i, _f]
    if hasattr(lib, "cOSSQS"):
        lib.cOSSQS.argtypes = [_fp] * 6 + [_f, _f, _i, _i] + fan[3:-1] + [_i, _f]
    return lib


def p(a):
    return a.ctypes.data_as(_fp)


FAN_CASES = {
    # name: geometry, batches, channels, nview
    "fan2d": (dict(nx=48, ny=40, nz=1, dx=1.0, dy=1.1, dz=1.0, nu=64, nv=1, da=0.0025, dv=1.0, off_a=0.0,
                   off_v=0.0, dsd=1085.6, dso=595.0), 1, 1, 72),
    "fan_offsets": (dict(nx=40, ny=52, nz=1, dx=0.9, dy=1.0, dz=1.0, nu=64, nv=1, da=0.0025, dv=1.0, off_a=0.7,
                         off_v=0.0, dsd=1085.6, dso=595.0), 1, 1, 45),
    "fan_multislice": (dict(nx=48, ny=40, nz=3, dx=1.0, dy=1.1, dz=1.0, nu=64, nv=3, da=0.0025, dv=1.0, off_a=0.0,
                            off_v=0.0, dsd=1085.6, dso=595.0), 2, 2, 36),
    "fan256": (dict(nx=256, ny=256, nz=1, dx=1.0, dy=1.0, dz=1.0, nu=736, nv=1, da=1.2858 / 1085.6, dv=1.0,
                      off_a=0.0, off_v=0.0, dsd=1085.6, dso=595.0), 1, 1, 45),
}


def fan_case(lib, name, rng):
    g, B, C, nview = FAN_CASES[name]
    ang = (np.arange(nview) * 2 * np.pi / nview).astype(np.float32)
    img = rng.random((B, g["nx"], g["ny"], g["nz"], C)).astype(np.float32)
    sino_in = rng.random((B, g["nu"], nview, g["nv"], C)).astype(np.float32)
    args = lambda t: (B, C, g["nx"], g["ny"], g["nz"], g["dx"], g["dy"], g["dz"], g["nu"], nview, g["nv"], g["da"],
                      g["dv"], g["off_a"], g["off_v"], g["dsd"], g["dso"], t)
    fp = np.zeros((B, g["nu"], nview, g["nv"], C), np.float32)
    lib.cDistanceDrivenFanProjection(p(fp), p(img), p(ang), *args(0))
    out = dict(img=img, sino_in=sino_in, angles=ang, fp=fp, B=B, C=C, **{k: np.float64(v) for k, v in g.items()})
    for t in (0, 1):
        bp = np.zeros(img.shape, np.float32)
        lib.cDistanceDrivenFanBackprojection(p(bp), p(sino_in), p(ang), *args(t))
        out[f"bp{t}"] = bp
    if g["nv"] == 1 and C == 1 and g["nx"] <= 64:
        for tf in (0, 2):
            fs = np.zeros(sino_in.shape, np.float32)
            lib.cFilterFanFilter(p(fs), p(sino_in), B, C, g["nu"], nview, g["nv"], g["da"], g["dv"], g["off_a"],
                                 g["off_v"], g["dsd"], g["dso"], tf, 1)
            out[f"filt{tf}"] = fs
    return out


def tv_case(lib, rng):
    img = (rng.random((1, 37, 29, 1)) * 0.02).astype(np.float32)
    grad = np.zeros_like(img)
    norm = np.zeros_like(img)
    tv = lib.cTVSQS2D(p(grad), p(norm), p(img), 37, 29)
    return dict(img=img, grad=grad, norm=norm, tv=np.float64(tv))


def tomo_case(lib, rng):
    nview = 5
    dc = np.zeros((nview, 3), np.float32)
    src = np.zeros((nview, 3), np.float32)
    for k in range(nview):
        a = (k - (nview - 1) / 2) * 0.15
        src[k] = (600 * math.sin(a), 10.0, 600 * math.cos(a))
        dc[k] = (0.0, 0.0, -40.0)
    g = dict(dx=1.0, dy=1.0, dz=2.0, cx=0.0, cy=0.0, cz=0.0, du=1.5, dv=1.5, off_u=0.2, off_v=-0.3)
    nx, ny, nz, nu, nv = 16, 14, 6, 24, 20
    img = rng.random((1, nx, ny, nz, 1)).astype(np.float32)
    prj_in = rng.random((1, nu, nview, nv, 1)).astype(np.float32)
    targs = (1, 1, nx, ny, nz, g["dx"], g["dy"], g["dz"], g["cx"], g["cy"], g["cz"], nu, nview, nv, g["du"],
             g["dv"], g["off_u"], g["off_v"])
    fp = np.zeros((1, nu, nview, nv, 1), np.float32)
    lib.cDistanceDrivenTomoProjection(p(fp), p(img), p(dc), p(src), *targs)
    bp = np.zeros(img.shape, np.float32)
    lib.cDistanceDrivenTomoBackprojection(p(bp), p(prj_in), p(dc), p(src), *targs)
    return dict(img=img, prj_in=prj_in, det_center=dc, src=src, fp=fp, bp=bp, nu=nu, nv=nv,
                **{k: np.float64(v) for k, v in g.items()})


SIDDON_CASES = {
    "siddon2d": (dict(nx=48, ny=40, nz=1, dx=1.0, dy=1.1, dz=1.0, nu=64, nv=1, da=0.0025, dv=1.0, off_a=0.3,
                      off_v=0.0, dsd=1085.6, dso=595.0), 1, 1, 72),
    "siddon_multislice": (dict(nx=40, ny=36, nz=3, dx=1.0, dy=1.0, dz=1.0, nu=48, nv=3, da=0.003, dv=1.0,
                               off_a=0.0, off_v=0.25, dsd=1085.6, dso=595.0), 2, 1, 30),
}


def siddon_case(lib, rng):
    """cSiddonFanProjection / cSiddonFanBackprojection (Siddon.cu:424-538)."""
    out = {}
    for name, (g, B, C, nview) in SIDDON_CASES.items():
        ang = (np.arange(nview) * 2 * np.pi / nview + 0.013).astype(np.float32)
        img = rng.random((B, g["nx"], g["ny"], g["nz"], C)).astype(np.float32)
        sino_in = rng.random((B, g["nu"], nview, g["nv"], C)).astype(np.float32)
        args = (B, C, g["nx"], g["ny"], g["nz"], g["dx"], g["dy"], g["dz"], g["nu"], nview, g["nv"], g["da"], g["dv"],
                g["off_a"], g["off_v"], g["dsd"], g["dso"], 0)
        fp = np.zeros((B, g["nu"], nview, g["nv"], C), np.float32)
        lib.cSiddonFanProjection(p(fp), p(img), p(ang), *args)
        bp = np.zeros(img.shape, np.float32)
        lib.cSiddonFanBackprojection(p(bp), p(sino_in), p(ang), *args)
        out[name] = dict(img=img, sino_in=sino_in, angles=ang, fp=fp, bp=bp, B=B, C=C,
                         **{k: np.float64(v) for k, v in g.items()})
    return out


PIXEL_CASES = {
    "pixel2d": (dict(nx=48, ny=40, nz=1, dx=1.0, dy=1.1, dz=1.0, nu=64, nv=1, da=0.0025, dv=1.0, off_a=0.3,
                     off_v=0.0, dsd=1085.6, dso=595.0), 2, 72),
    # slices between detector rows (v interpolation) and rows beyond the volume
    "pixel_multislice": (dict(nx=40, ny=36, nz=3, dx=1.0, dy=1.0, dz=1.3, nu=48, nv=4, da=0.003, dv=1.0,
                              off_a=-0.4, off_v=0.35, dsd=1085.6, dso=595.0), 1, 30),
}


def pixel_case(lib, rng):
    """cPixelDrivenFanBackprojection (PixelDriven.cu:100-141), nChannels = 1."""
    out = {}
    for name, (g, B, nview) in PIXEL_CASES.items():
        ang = (np.arange(nview) * 2 * np.pi / nview + 0.021).astype(np.float32)
        sino_in = rng.random((B, g["nu"], nview, g["nv"], 1)).astype(np.float32)
        args = (B, 1, g["nx"], g["ny"], g["nz"], g["dx"], g["dy"], g["dz"], g["nu"], nview, g["nv"], g["da"], g["dv"],
                g["off_a"], g["off_v"], g["dsd"], g["dso"], 0)
        bp = np.zeros((B, g["nx"], g["ny"], g["nz"], 1), np.float32)
        lib.cPixelDrivenFanBackprojection(p(bp), p(sino_in), p(ang), *args)
        out[name] = dict(sino_in=sino_in, angles=ang, bp=bp, B=B, **{k: np.float64(v) for k, v in g.items()})
    return out


def cone_geometry(name):
    """Grid, detector and per-view geometry ([nview, 3] arrays, mm) of the
    cone test cases: a tomosynthesis arc (rays mostly along z), a circular
    cone-beam scan whose views cross 45 degrees (the main axis switches
    between x and y), and a tilted, off-centre detector."""
    if name == "cone_tomo":
        g = dict(nx=14, ny=12, nz=6, dx=1.0, dy=0.9, dz=1.5, cx=0.4, cy=-0.3, cz=0.2, nu=20, nv=18, du=1.2,
                 dv=1.1, off_u=0.3, off_v=-0.4)
        nview = 7
        src = np.zeros((nview, 3), np.float32)
        dc = np.zeros((nview, 3), np.float32)
        for k in range(nview):
            a = (k - (nview - 1) / 2) * 0.12
            src[k] = (400 * math.sin(a), 6.0, 400 * math.cos(a))
            dc[k] = (1.0, -0.5, -30.0)
        du = np.tile(np.float32([1, 0, 0]), (nview, 1))
        dv = np.tile(np.float32([0, 1, 0]), (nview, 1))
    elif name == "cone_circular":
        g = dict(nx=12, ny=13, nz=5, dx=1.0, dy=1.0, dz=1.2, cx=0.0, cy=0.5, cz=-0.3, nu=24, nv=8, du=1.5,
                 dv=1.4, off_u=0.2, off_v=0.1)
        nview = 9
        ang = np.arange(nview) * (2 * np.pi / nview) + np.pi / 4 - 0.01
        src = np.stack([300 * np.cos(ang), 300 * np.sin(ang), np.full(nview, 1.0)], 1).astype(np.float32)
        dc = np.stack([-250 * np.cos(ang), -250 * np.sin(ang), np.full(nview, 1.0)], 1).astype(np.float32)
        du = np.stack([-np.sin(ang), np.cos(ang), np.zeros(nview)], 1).astype(np.float32)
        dv = np.tile(np.float32([0, 0, 1]), (nview, 1))
    else:   # cone_tilted
        g = dict(nx=10, ny=11, nz=9, dx=1.1, dy=1.0, dz=0.9, cx=0.0, cy=0.0, cz=0.0, nu=16, nv=15, du=1.4,
                 dv=1.3, off_u=-0.6, off_v=0.25)
        nview = 5
        src = np.zeros((nview, 3), np.float32)
        dc = np.zeros((nview, 3), np.float32)
        du = np.zeros((nview, 3), np.float32)
        dv = np.zeros((nview, 3), np.float32)
        for k in range(nview):
            t = 0.3 * (k - 2)
            src[k] = (50 * math.sin(t), 320 * math.cos(0.2 * k), 20.0)
            dc[k] = (-3.0, -150.0, -10.0)
            # u mostly along x, v mostly along z: the plane faces the source (y)
            u = np.array([math.cos(0.15), 0.05, math.sin(0.15)])
            u /= np.linalg.norm(u)
            v = np.cross(u, np.array([0.1, 1.0, 0.05]))
            du[k] = u
            dv[k] = v / np.linalg.norm(v)
    return g, dc, du, dv, src


CONE_CASES = ("cone_tomo", "cone_circular", "cone_tilted")


def cone_case(lib, rng):
    """cSiddonConeProjectionAbitrary / ...BackprojectionAbitrary
    (SiddonCone.cu:126-278) and cOSSQSConeAbitrary (ossqs.cu:163-333)."""
    out = {}
    for name in CONE_CASES:
        g, dc, du, dv, src = cone_geometry(name)
        nview = dc.shape[0]
        img = rng.random((1, g["nx"], g["ny"], g["nz"], 1)).astype(np.float32)
        prj_in = rng.random((1, g["nu"], nview, g["nv"], 1)).astype(np.float32)
        args = (1, 1, g["nx"], g["ny"], g["nz"], g["dx"], g["dy"], g["dz"], g["cx"], g["cy"], g["cz"], g["nu"], nview,
                g["nv"], g["du"], g["dv"], g["off_u"], g["off_v"])
        fp = np.zeros((1, g["nu"], nview, g["nv"], 1), np.float32)
        lib.cSiddonConeProjectionAbitrary(p(fp), p(img), p(dc), p(du), p(dv), p(src), *args)
        bp = np.zeros(img.shape, np.float32)
        lib.cSiddonConeBackprojectionAbitrary(p(bp), p(prj_in), p(dc), p(du), p(dv), p(src), *args)
        d = dict(img=img, prj_in=prj_in, det_center=dc, det_u=du, det_v=dv, src=src, fp=fp, bp=bp,
                 **{k: np.float64(v) for k, v in g.items()})
        if name == "cone_tomo" and hasattr(lib, "cOSSQSConeAbitrary"):
            # one OS-SQS pass: 7 subsets of one view, a mask and a clamp
            norm = np.zeros(img.shape, np.float32)
            ones = np.ones(img.shape, np.float32)
            a1 = np.zeros(fp.shape, np.float32)
            lib.cSiddonConeProjectionAbitrary(p(a1), p(ones), p(dc), p(du), p(dv), p(src), *args)
            lib.cSiddonConeBackprojectionAbitrary(p(norm), p(a1), p(dc), p(du), p(dv), p(src), *args)
            mask = (rng.random(img.shape) > 0.1).astype(np.float32)
            x0 = (rng.random(img.shape) * 0.5).astype(np.float32)
            res = np.zeros(img.shape, np.float32)
            lib.cOSSQSConeAbitrary(p(res), p(x0), p(fp), p(norm), p(mask), p(dc), p(du), p(dv), p(src), 0.0, 1.0,
                                   1, nview, *args, 2, 0.7)
            d.update(ossqs_x0=x0, ossqs_norm=norm, ossqs_mask=mask, ossqs_res=res, ossqs_lam=0.7)
        out[name] = d
    return out


PRIOR_REF = os.path.join(ROOT, "oracle", "_ref", "libprior_ref.so")


def load_prior_ref(path=PRIOR_REF):
    lib = ctypes.CDLL(path)
    lib.cTVSQS2D.argtypes = [_fp, _fp, _fp, _fp, _i, _i, _i, _i, _f]
    lib.cTVSQS3D.argtypes = [_fp, _fp, _fp, _fp, _i, _i, _i, _i, _i, _f]
    return lib


def prior_case(lib, rng):
    """cTVSQS2D / cTVSQS3D of the prior solver (PriorFunctionSolver/TVSQS.cu):
    smooth-plus-noise images with flat patches (zero differences, where eps
    matters), two batches and two channels."""
    out = {}
    for ndim, shape in ((2, (2, 23, 17, 2)), (3, (2, 11, 9, 7, 2))):
        x = rng.random(shape).astype(np.float32)
        x[0, 2:6, 3:8] = 0.5
        s1, s2, var = (np.zeros(shape, np.float32) for _ in range(3))
        if ndim == 2:
            lib.cTVSQS2D(p(s1), p(s2), p(var), p(x), *shape, 1e-8)
        else:
            lib.cTVSQS3D(p(s1), p(s2), p(var), p(x), *shape, 1e-8)
        out[f"tviso{ndim}d"] = dict(img=x, s1=s1, s2=s2, var=var, ndim=ndim, eps=1e-8)
    return out


def ossqs_case(lib, rng):
    """cOSSQS (ossqs.cu:12-161, the Siddon pair): a 2D slice, 60 views in 4
    contiguous subsets of 15 (nview a multiple of nviewPerSubset, so the
    reference's tail-subset rule does not come into play), weights in
    [0.5, 1.5), a clamp to [0, 1], lambda 0.8, one pass."""
    g = dict(SIDDON_CASES["siddon2d"][0])
    nview, M = 60, 4
    ang = (np.arange(nview) * 2 * np.pi / nview + 0.013).astype(np.float32)
    truth = (rng.random((1, g["nx"], g["ny"], 1, 1)) * 0.02).astype(np.float32)
    args = (1, 1, g["nx"], g["ny"], g["nz"], g["dx"], g["dy"], g["dz"], g["nu"], nview, g["nv"], g["da"], g["dv"],
            g["off_a"], g["off_v"], g["dsd"], g["dso"])
    sino = np.zeros((1, g["nu"], nview, 1, 1), np.float32)
    lib.cSiddonFanProjection(p(sino), p(truth), p(ang), *args, 0)
    w = (0.5 + rng.random(sino.shape)).astype(np.float32)
    ones = np.ones(truth.shape, np.float32)
    a1 = np.zeros(sino.shape, np.float32)
    lib.cSiddonFanProjection(p(a1), p(ones), p(ang), *args, 0)
    a1 = np.ascontiguousarray(a1 * w)
    norm = np.zeros(truth.shape, np.float32)
    lib.cSiddonFanBackprojection(p(norm), p(a1), p(ang), *args, 0)
    x0 = (rng.random(truth.shape) * 0.02).astype(np.float32)
    res = np.zeros(truth.shape, np.float32)
    lib.cOSSQS(p(res), p(x0), p(sino), p(norm), p(w), p(ang), 0.0, 1.0, nview // M, M, *args, 0, 0.8)
    return dict(x0=x0, sino=sino, w=w, norm=norm, angles=ang, res=res, n_subsets=M, lam=0.8, lb=0.0, ub=1.0,
                **{k: np.float64(v) for k, v in g.items()})


def main(outdir=HERE, only=None):
    if only == "siddon":
        lib = load_ref()
        for name, d in siddon_case(lib, np.random.default_rng(20241203)).items():
            np.savez_compressed(os.path.join(outdir, f"ref_{name}.npz"), **d)
        print("siddon golden vectors written to", outdir)
        return
    if only == "pixel":
        lib = load_ref()
        for name, d in pixel_case(lib, np.random.default_rng(20241205)).items():
            np.savez_compressed(os.path.join(outdir, f"ref_{name}.npz"), **d)
        print("pixel-driven golden vectors written to", outdir)
        return
    if only == "cone":
        lib = load_ref()
        for name, d in cone_case(lib, np.random.default_rng(20241207)).items():
            np.savez_compressed(os.path.join(outdir, f"ref_{name}.npz"), **d)
        print("cone golden vectors written to", outdir)
        return
    if only == "prior":
        lib = load_prior_ref()
        for name, d in prior_case(lib, np.random.default_rng(20241206)).items():
            np.savez_compressed(os.path.join(outdir, f"ref_{name}.npz"), **d)
        print("prior-solver golden vectors written to", outdir)
        return
    if only == "ossqs":
        lib = load_ref()
        np.savez_compressed(os.path.join(outdir, "ref_ossqs_siddon.npz"),
                            **ossqs_case(lib, np.random.default_rng(20241204)))
        print("cOSSQS golden vectors written to", outdir)
        return
    lib = load_ref()
    rng = np.random.default_rng(20240601)
    for name in FAN_CASES:
        np.savez_compressed(os.path.join(outdir, f"ref_{name}.npz"), **fan_case(lib, name, rng))
    np.savez_compressed(os.path.join(outdir, "ref_tv.npz"), **tv_case(lib, rng))
    np.savez_compressed(os.path.join(outdir, "ref_tomo.npz"), **tomo_case(lib, rng))
    print("golden vectors written to", outdir)


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    only = next((k for k in ("siddon", "ossqs", "pixel", "prior", "cone") if f"--{k}" in sys.argv), None)
    main(args[0] if args else HERE, only=only)
