"""TEST INFRASTRUCTURE -- the CPU oracle for the DD hot path (not product code).

ctypes wrapper over ``oracle/liboracle.so`` (built from ``oracle/oracle.cpp`` by
``oracle/Makefile``).  Only ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline / reference legs of ``bench.py`` may import this module.

Array conventions are the reference's (python/ReconNet_no_tf.py:133-200):
images are ``[B, nx, ny, nz, C]`` and sinograms ``[B, nu, nview, nv, C]``, C-order.
Geometry objects only need the attributes ``dx dy dz da dv off_a off_v dsd dso``
(fan) or ``dx dy dz cx cy cz du dv off_u off_v`` (tomo).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

_f = ctypes.c_float
_i = ctypes.c_int
_fp = ctypes.POINTER(ctypes.c_float)
_dp = ctypes.POINTER(ctypes.c_double)

_FAN = [_i, _i, _i, _i, _i, _f, _f, _f, _i, _i, _i, _f, _f, _f, _f, _f, _f]
_TOMO = [_i, _i, _i, _i, _i, _f, _f, _f, _f, _f, _f, _i, _i, _i, _f, _f, _f, _f]
_CYL = [_i, _i, _i, _i, _f, _f, _f, _f, _f, _f, _i, _i, _i, _f, _f, _f, _f, _f, _f]


def build(force: bool = False) -> str:
    """Compile liboracle.so with the committed Makefile (gcc, OpenMP)."""
    src = os.path.join(_HERE, "oracle.cpp")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", _HERE, "liboracle.so"])
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        L.oracle_num_threads.restype = _i
        L.oracle_set_num_threads.argtypes = [_i]
        L.oracle_view_is_x.argtypes = [_f]
        L.oracle_view_is_x.restype = _i
        L.oracle_set_tex_quant.argtypes = [_i]
        L.oracle_fan_fp_f64.argtypes = [_dp, _fp, _fp] + _FAN
        L.oracle_fan_fp_f32.argtypes = [_fp, _fp, _fp] + _FAN
        L.oracle_fan_bp_f64.argtypes = [_dp, _fp, _fp] + _FAN + [_i]
        L.oracle_siddon_fp_f64.argtypes = [_dp, _fp, _fp] + _FAN
        L.oracle_siddon_bp_f64.argtypes = [_dp, _fp, _fp] + _FAN
        L.oracle_pixel_bp_f64.argtypes = [_dp, _fp, _fp] + _FAN
        L.oracle_pixel_bp_f32.argtypes = [_fp, _fp, _fp] + _FAN
        L.oracle_fan_bp_f32.argtypes = [_fp, _fp, _fp] + _FAN + [_i]
        L.oracle_ramp_kernel.argtypes = [_dp, _i, _f, _i, _i]
        L.oracle_filter_f64.argtypes = [_dp, _fp, _i, _i, _i, _i, _i, _f, _f, _f, _f, _f, _f, _i, _i]
        L.oracle_tv_sqs_f64.argtypes = [_dp, _dp, _fp, _i, _i]
        L.oracle_tv_sqs_f64.restype = ctypes.c_double
        L.oracle_tv_iso_sqs_f64.argtypes = [_dp, _dp, _dp, _fp, _i, _i, _i, _i, _i, ctypes.c_double, _i]
        L.oracle_cone_fp_f64.argtypes = [_dp, _fp, _fp, _fp, _fp, _fp] + _TOMO
        L.oracle_cone_bp_f64.argtypes = [_dp, _fp, _fp, _fp, _fp, _fp] + _TOMO
        L.oracle_tomo_fp_f64.argtypes = [_dp, _fp, _fp, _fp] + _TOMO
        L.oracle_tomo_bp_f64.argtypes = [_dp, _fp, _fp, _fp] + _TOMO + [_i]
        L.oracle_tex_fetch.argtypes = [_dp, _fp, _i, _i, _i, _i, _i, _i, _fp, _i]
        L.oracle_cyl_fp_f64.argtypes = [_dp, _fp, _fp] + _CYL
        L.oracle_cyl_fp_f32.argtypes = [_fp, _fp, _fp] + _CYL
        L.oracle_cyl_bp_f64.argtypes = [_dp, _fp, _fp] + _CYL
        _lib = L
    return _lib


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _ptr(a, t):
    return a.ctypes.data_as(ctypes.POINTER(t))


def set_threads(n: int) -> None:
    lib().oracle_set_num_threads(int(n))


def num_threads() -> int:
    return int(lib().oracle_num_threads())


def set_tex_quant(mode: int) -> None:
    """0 exact texture weights (default), 1 rounded / 2 truncated to 1/256."""
    lib().oracle_set_tex_quant(int(mode))


def tex_fetch(table, modes, coords, quant=3):
    """Linear-filtered fetches of the emulated texture unit: table [D, H, W],
    modes (border 0 / clamp 1) per dimension (w, h, d), coords [n, 3]."""
    t = _f32(table)
    c = _f32(coords)
    D, H, W = t.shape
    out = np.zeros(c.shape[0], np.float64)
    set_tex_quant(quant)
    try:
        lib().oracle_tex_fetch(_ptr(out, ctypes.c_double), _ptr(t, _f), W, H, D, *modes, _ptr(c, _f), c.shape[0])
    finally:
        set_tex_quant(0)
    return out


def view_is_x(deg: float) -> bool:
    return bool(lib().oracle_view_is_x(float(deg)))


def _fan_args(g, img_shape, sino_shape):
    B, nx, ny, nz, C = img_shape
    _, nu, nview, nv, _ = sino_shape
    return (B, C, nx, ny, nz, g.dx, g.dy, g.dz, nu, nview, nv, g.da, g.dv, g.off_a, g.off_v, g.dsd, g.dso)


def fan_fp(img, angles, g, nu, nv=None, dtype=np.float64):
    """DD fan forward projection (DistanceDriven.cu:64-384), exact texture lerp."""
    img = _f32(img)
    ang = _f32(angles)
    B, nx, ny, nz, C = img.shape
    nv = nz if nv is None else nv
    out = np.zeros((B, nu, ang.size, nv, C), dtype=dtype)
    args = _fan_args(g, img.shape, out.shape)
    if dtype == np.float64:
        lib().oracle_fan_fp_f64(_ptr(out, ctypes.c_double), _ptr(img, _f), _ptr(ang, _f), *args)
    else:
        lib().oracle_fan_fp_f32(_ptr(out, _f), _ptr(img, _f), _ptr(ang, _f), *args)
    return out


def fan_bp(sino, angles, g, img_shape, type_projector=0, dtype=np.float64):
    """DD fan backprojection.  type 0/1: reference DDBPFanKernelX/Y
    (DistanceDriven.cu:441-791); type 2: exact transpose of ``fan_fp``."""
    sino = _f32(sino)
    ang = _f32(angles)
    B, nu, nview, nv, C = sino.shape
    nx, ny, nz = img_shape
    out = np.zeros((B, nx, ny, nz, C), dtype=dtype)
    args = _fan_args(g, out.shape, sino.shape)
    if dtype == np.float64:
        lib().oracle_fan_bp_f64(_ptr(out, ctypes.c_double), _ptr(sino, _f), _ptr(ang, _f), *args, int(type_projector))
    else:
        lib().oracle_fan_bp_f32(_ptr(out, _f), _ptr(sino, _f), _ptr(ang, _f), *args, int(type_projector))
    return out


def ramp_kernel(nu, da, type_filter=0, equispace=False):
    """Spatial filter kernel of getRamp (Filter.cu:66-214), length 2nu-1."""
    h = np.zeros(2 * nu - 1, np.float64)
    lib().oracle_ramp_kernel(_ptr(h, ctypes.c_double), int(nu), float(da), int(type_filter), int(bool(equispace)))
    return h


def siddon_fp(img, angles, g, nu, nv=None):
    """Siddon fan forward projection (Siddon.cu:14-266): ray lengths in mm
    through each voxel, exact FP64 crossings."""
    img = _f32(img)
    ang = _f32(angles)
    B, nx, ny, nz, C = img.shape
    nv = nz if nv is None else nv
    out = np.zeros((B, nu, ang.size, nv, C), np.float64)
    lib().oracle_siddon_fp_f64(_ptr(out, ctypes.c_double), _ptr(img, _f), _ptr(ang, _f),
                               *_fan_args(g, img.shape, out.shape))
    return out


def siddon_bp(sino, angles, g, img_shape):
    """Transpose of ``siddon_fp`` (Siddon.cu:268-420 scatters with atomics)."""
    sino = _f32(sino)
    ang = _f32(angles)
    B, nu, nview, nv, C = sino.shape
    nx, ny, nz = img_shape
    out = np.zeros((B, nx, ny, nz, C), np.float64)
    lib().oracle_siddon_bp_f64(_ptr(out, ctypes.c_double), _ptr(sino, _f), _ptr(ang, _f),
                               *_fan_args(g, out.shape, sino.shape))
    return out


def pixel_bp(sino, angles, g, img_shape, dtype=np.float64):
    """Pixel-driven fan backprojection with the FBP weight
    (PixelDriven.cu:11-97); the output is overwritten."""
    sino = _f32(sino)
    ang = _f32(angles)
    B, nu, nview, nv, C = sino.shape
    nx, ny, nz = img_shape
    out = np.zeros((B, nx, ny, nz, C), dtype=dtype)
    args = _fan_args(g, out.shape, sino.shape)
    if dtype == np.float64:
        lib().oracle_pixel_bp_f64(_ptr(out, ctypes.c_double), _ptr(sino, _f), _ptr(ang, _f), *args)
    else:
        lib().oracle_pixel_bp_f32(_ptr(out, _f), _ptr(sino, _f), _ptr(ang, _f), *args)
    return out


def filter_sino(sino, g, type_filter=0, fan=True):
    """cFilterFan::Filter / cFilterParallel::Filter (Filter.cu:216-430)."""
    sino = _f32(sino)
    B, nu, nview, nv, C = sino.shape
    out = np.zeros(sino.shape, np.float64)
    lib().oracle_filter_f64(_ptr(out, ctypes.c_double), _ptr(sino, _f), B, C, nu, nview, nv, g.da, g.dv, g.off_a,
                            g.off_v, g.dsd, g.dso, int(type_filter), int(bool(fan)))
    return out


def tv_sqs(img2d):
    """TVSQSKernel + cTVSQS2D (TotalVariation.cu:9-142); img2d is [nx, ny]."""
    img = _f32(img2d)
    nx, ny = img.shape
    grad = np.zeros((nx, ny), np.float64)
    norm = np.zeros((nx, ny), np.float64)
    tv = lib().oracle_tv_sqs_f64(_ptr(grad, ctypes.c_double), _ptr(norm, ctypes.c_double), _ptr(img, _f), nx, ny)
    return grad, norm, float(tv)


def tv_iso_sqs(img, ndim, eps=1e-8):
    """Isotropic TV surrogate (PriorFunctionSolver/TVSQS.cu:8-93, 160-265):
    img is [nb, nx, ny, nc] (ndim 2) or [nb, nx, ny, nz, nc] (ndim 3);
    returns (s1, s2, var) in FP64."""
    img = _f32(img)
    if ndim == 2:
        nb, nx, ny, nc = img.shape
        nz = 1
    else:
        nb, nx, ny, nz, nc = img.shape
    s1, s2, var = (np.zeros(img.shape, np.float64) for _ in range(3))
    d = ctypes.c_double
    lib().oracle_tv_iso_sqs_f64(_ptr(s1, d), _ptr(s2, d), _ptr(var, d), _ptr(img, _f), nb, nx, ny, nz, nc,
                                float(eps), int(ndim))
    return s1, s2, var


def cone_fp(img, det_center, det_u, det_v, src, g, nu, nv):
    """Siddon cone projection, arbitrary geometry (SiddonCone.cu:20-42)."""
    img = _f32(img)
    B, nx, ny, nz, C = img.shape
    geo = [_f32(a).reshape(-1, 3) for a in (det_center, det_u, det_v, src)]
    out = np.zeros((B, nu, geo[0].shape[0], nv, C), np.float64)
    lib().oracle_cone_fp_f64(_ptr(out, ctypes.c_double), _ptr(img, _f), *[_ptr(a, _f) for a in geo],
                             *_tomo_args(g, img.shape, out.shape))
    return out


def cone_bp(prj, det_center, det_u, det_v, src, g, img_shape):
    """Transpose of ``cone_fp`` (SiddonCone.cu:44-67 scatters with atomics)."""
    prj = _f32(prj)
    B, nu, nview, nv, C = prj.shape
    nx, ny, nz = img_shape
    geo = [_f32(a).reshape(-1, 3) for a in (det_center, det_u, det_v, src)]
    out = np.zeros((B, nx, ny, nz, C), np.float64)
    lib().oracle_cone_bp_f64(_ptr(out, ctypes.c_double), _ptr(prj, _f), *[_ptr(a, _f) for a in geo],
                             *_tomo_args(g, out.shape, prj.shape))
    return out


def _tomo_args(g, img_shape, prj_shape):
    B, nx, ny, nz, C = img_shape
    _, nu, nview, nv, _ = prj_shape
    return (B, C, nx, ny, nz, g.dx, g.dy, g.dz, g.cx, g.cy, g.cz, nu, nview, nv, g.du, g.dv, g.off_u, g.off_v)


def tomo_fp(img, det_center, src, g, nu, nv):
    """DistanceDrivenTomo::ProjectionTomo (DistanceDriven3D.cu:139-343)."""
    img = _f32(img)
    dc = _f32(det_center)
    sp = _f32(src)
    B, nx, ny, nz, C = img.shape
    out = np.zeros((B, nu, dc.shape[0], nv, C), np.float64)
    lib().oracle_tomo_fp_f64(_ptr(out, ctypes.c_double), _ptr(img, _f), _ptr(dc, _f), _ptr(sp, _f),
                             *_tomo_args(g, img.shape, out.shape))
    return out


def tomo_bp(prj, det_center, src, g, img_shape, weight_mode=0):
    """DistanceDrivenTomo::BackprojectionTomo (DistanceDriven3D.cu:409-663).

    weight_mode 0 reproduces the reference (length pre-weight on view 0 only,
    DistanceDriven3D.cu:612-621); 1 weights every view."""
    prj = _f32(prj)
    dc = _f32(det_center)
    sp = _f32(src)
    B, nu, nview, nv, C = prj.shape
    nx, ny, nz = img_shape
    out = np.zeros((B, nx, ny, nz, C), np.float64)
    lib().oracle_tomo_bp_f64(_ptr(out, ctypes.c_double), _ptr(prj, _f), _ptr(dc, _f), _ptr(sp, _f),
                             *_tomo_args(g, out.shape, prj.shape), int(weight_mode))
    return out


# ---------------------------------------------------------------------------
# OS-SQS composition (ossqs.cu:91-149 arithmetic with the DD projector, a TV
# term from TotalVariation.cu, explicit subset view lists).
# ---------------------------------------------------------------------------
def sqs_subset_update(x, sino, wsino, norm_img, angles, views, g, n_subsets, lam=1.0, beta=0.0,
                      lb=-np.inf, ub=np.inf, bp_type=2, projector="dd", dtype=np.float64):
    """One ordered-subset SQS step on a [nx, ny] slice (2D, B = C = 1),
    ossqs.cu:91-149 with the TV terms of the TV-regularised variant.

    x_new = clamp(x - lam * (M * A_s^T W_s (A_s x - b_s) + beta * grad_tv(x))
                        / (norm_img + beta * norm_tv(x) + 1e-6), lb, ub)
    ``sino``/``wsino`` are [nu, nview]; ``views`` lists the subset's view
    indices.  projector "dd": DD forward and the ``bp_type`` backprojector;
    "siddon": the Siddon pair (the reference cOSSQS projector, ossqs.cu:81).
    """
    x = np.asarray(x, np.float32)
    nx, ny = x.shape
    nu = sino.shape[0]
    views = np.asarray(views)
    ang = np.asarray(angles, np.float32)[views]
    if projector == "siddon":
        fp = siddon_fp(x[None, :, :, None, None], ang, g, nu, 1)[0, :, :, 0, 0]
    else:
        fp = fan_fp(x[None, :, :, None, None], ang, g, nu, 1, dtype=dtype)[0, :, :, 0, 0]
    r = (fp - sino[:, views].astype(np.float64)) * wsino[:, views].astype(np.float64)
    r = r.astype(np.float32)[None, :, :, None, None]
    if projector == "siddon":
        bp = siddon_bp(r, ang, g, (nx, ny, 1))[0, :, :, 0, 0]
    else:
        bp = fan_bp(r, ang, g, (nx, ny, 1), bp_type, dtype=dtype)[0, :, :, 0, 0]
    num = n_subsets * bp
    den = np.asarray(norm_img, np.float64) + 1e-6
    if beta > 0:
        grad, norm, _ = tv_sqs(x)
        num = num + beta * grad
        den = den + beta * norm
    xn = x.astype(np.float64) - lam * num / den
    return np.clip(xn, lb, ub)


def shortscan_weights(angles, nu, da, off_a, kind="parker", sigma=30.0, theta=10 * np.pi / 180, mask_all=False):
    """Short-scan redundancy weights [nu, nview] in FP64 with the reference's
    conventions (python/ReconNet_no_tf.py:640-693): channel angle
    alpha = ((u - (nu-1)/2) - off_a) * da, half over-scan
    gamma = (angles[-1] - pi) / 2.

    Parker (Med. Phys. 9(2), 1982): sin^2 ramps over the doubly measured
    wedges beta < 2(gamma - alpha) and beta > pi - 2 alpha, 1 between.
    Riess: the ramps continued past those wedges as 2 - ramp (reference
    precedence :681-684: first wedge, its continuation, second wedge, its
    continuation), rounded to FP32 as the reference stores them, then smoothed
    along the channels by a normalised Gaussian of `sigma` channels reaching
    int(4 sigma + 0.5) channels with edge values repeated -- except, in views
    with theta < beta < pi + 2 gamma - theta, channel 0 (the reference's
    np.where over the 0-d result of np.all, :687-688) or, with mask_all, the
    whole view."""
    ang = np.asarray(angles, np.float32).astype(np.float64)
    beta = ang[None, :]
    gamma = (ang[-1] - np.pi) / 2
    alpha = ((np.arange(nu) - (nu - 1) / 2.0) - off_a)[:, None] * float(da)
    with np.errstate(divide="ignore", invalid="ignore"):
        ramp_in = np.sin(np.pi / 4 * beta / (gamma - alpha)) ** 2
        ramp_out = np.sin(np.pi / 4 * (np.pi + 2 * gamma - beta) / (gamma + alpha)) ** 2
    first_wedge = beta < 2 * gamma - 2 * alpha
    if kind == "parker":
        return np.where(first_wedge, ramp_in, np.where(beta <= np.pi - 2 * alpha, 1.0, ramp_out))
    conds = [first_wedge, beta < -2 * gamma + 2 * alpha, beta > np.pi - 2 * alpha, beta > np.pi + 2 * gamma + 2 * alpha]
    vals = [ramp_in, 2 - ramp_in, ramp_out, 2 - ramp_out]
    full = np.broadcast_shapes(alpha.shape, beta.shape)
    w = np.select([np.broadcast_to(c, full) for c in conds], [np.broadcast_to(v, full) for v in vals], default=1.0)
    w = w.astype(np.float32).astype(np.float64)
    r = int(4.0 * sigma + 0.5)
    taps = np.exp(-0.5 * (np.arange(-r, r + 1) / sigma) ** 2)
    taps /= taps.sum()
    padded = np.pad(w, ((r, r), (0, 0)), mode="edge")
    smooth = np.zeros_like(w)
    for k in range(2 * r + 1):
        smooth += taps[k] * padded[k:k + nu]
    keep_view = (beta > theta) & (beta < np.pi + 2 * gamma - theta)        # [1, nview]
    keep = np.broadcast_to(keep_view, full).copy()
    if not mask_all:
        keep[1:, :] = False
    return np.where(keep, w, smooth)


def _cyl_args(g, nb, vol_shape, nview):
    nx, ny, nz = vol_shape
    return (nb, nx, ny, nz, g.dx, g.dy, g.dz, g.cx, g.cy, g.cz, g.nu, nview, g.nv, g.da, g.dv, g.off_a, g.off_v,
            g.dsd, g.dso)


def cyl_fp(vol, angles, g, dtype=np.float64):
    """Cylindrical-detector cone-beam DD forward projection (definition in
    oracle.cpp, section "Cylindrical-detector cone-beam DD pair"): vol is
    [B, nx, ny, nz], returns [B, nu, nview, nv]."""
    vol = _f32(vol)
    ang = _f32(angles)
    B, nx, ny, nz = vol.shape
    out = np.zeros((B, g.nu, ang.size, g.nv), dtype)
    fn = lib().oracle_cyl_fp_f64 if dtype == np.float64 else lib().oracle_cyl_fp_f32
    ct = ctypes.c_double if dtype == np.float64 else _f
    fn(_ptr(out, ct), _ptr(vol, _f), _ptr(ang, _f), *_cyl_args(g, B, (nx, ny, nz), ang.size))
    return out


def cyl_bp(prj, angles, g, vol_shape):
    """Exact transpose of cyl_fp: prj [B, nu, nview, nv] -> [B, nx, ny, nz]."""
    prj = _f32(prj)
    ang = _f32(angles)
    B = prj.shape[0]
    out = np.zeros((B,) + tuple(vol_shape), np.float64)
    lib().oracle_cyl_bp_f64(_ptr(out, ctypes.c_double), _ptr(prj, _f), _ptr(ang, _f),
                            *_cyl_args(g, B, vol_shape, ang.size))
    return out


# ---- the learned prior's 3x3 convolutions (FP64 numpy) -------------------------
# Tap (dy, dx) of output pixel (h, w) reads input pixel (h + dy - 1, w + dx - 1),
# zero outside the image; weights are [cout, 3, 3, cin].

def bf16_round(a):
    """Round float32 values to bfloat16 (nearest even), returned as float64."""
    a = np.ascontiguousarray(a, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def conv3x3(x, w, b=None):
    """x [N, cin, H, W], w [cout, 3, 3, cin] -> [N, cout, H, W] in FP64."""
    x = np.asarray(x, np.float64)
    w = np.asarray(w, np.float64)
    N, C, H, W = x.shape
    xp = np.pad(x, ((0, 0), (0, 0), (1, 1), (1, 1)))
    y = np.zeros((N, w.shape[0], H, W))
    for dy in range(3):
        for dx in range(3):
            y += np.einsum("nchw,oc->nohw", xp[:, :, dy:dy + H, dx:dx + W], w[:, dy, dx, :], optimize=True)
    if b is not None:
        y += np.asarray(b, np.float64)[None, :, None, None]
    return y


def conv3x3_dgrad(dy, w):
    """Gradient with respect to the input: dy [N, cout, H, W] -> [N, cin, H, W]."""
    w = np.asarray(w, np.float64)
    return conv3x3(dy, w[:, ::-1, ::-1, :].transpose(3, 1, 2, 0))


def conv3x3_wgrad(x, dy):
    """Gradients with respect to the weights [cout, 3, 3, cin] and bias [cout]."""
    x = np.asarray(x, np.float64)
    dy = np.asarray(dy, np.float64)
    N, C, H, W = x.shape
    xp = np.pad(x, ((0, 0), (0, 0), (1, 1), (1, 1)))
    dw = np.zeros((dy.shape[1], 3, 3, C))
    for a in range(3):
        for c in range(3):
            dw[:, a, c, :] = np.einsum("nohw,nchw->oc", dy, xp[:, :, a:a + H, c:c + W], optimize=True)
    return dw, dy.sum(axis=(0, 2, 3))
