"""Host (numpy) API mirroring the reference's ``ReconNet`` class.

Same attribute names, defaults and method signatures as
python/ReconNet_no_tf.py:26-632 for the distance-driven path; every method
calls the reference-named C entry points of ``libreconnet_b200.so`` and raises
``ReconNetError`` on failure (the reference printed to stderr and threw).
"""
from __future__ import annotations

import ctypes
import re

import numpy as np

from . import _native as N

_c = ctypes


def _out(shape, dtype=np.float32):
    """Output array of a call that writes every element of it (the fan and
    tomosynthesis projections and backprojections: the library copies its
    whole device result into it).  Left uninitialised: filling a fresh array
    of a few MB with zeros first costs about as much as the call's own copies
    (its pages are faulted in and cleared), ~20% of a per-slice call pair."""
    return np.empty(shape, dtype)


def _fptr(a):
    return a.ctypes.data_as(_c.POINTER(_c.c_float))


class ReconNet:
    """Geometry holder + DD projector calls (python/ReconNet_no_tf.py:26)."""

    def __init__(self):
        # defaults of python/ReconNet_no_tf.py:27-47
        self.rotview = 720
        self.nu = 736
        self.nv = 1
        self.nx = 512
        self.ny = 512
        self.nz = 1
        self.dx = 1
        self.dy = 1
        self.dz = 2
        self.cx = 0
        self.cy = 0
        self.cz = 0
        self.dsd = 1085.6
        self.dso = 595
        self.du = 1.2858
        self.dv = 2
        self.da = self.du / self.dsd
        self.off_a = 0
        self.off_u = 0
        self.off_v = 0
        self.UpdateAngularSampling()

    def FromFile(self, filename):
        """Whitespace-separated ``name value`` lines (ReconNet_no_tf.py:49-73)."""
        params = {}
        with open(filename, "r") as f:
            for line in f:
                parts = [p for p in re.split(r"[ \t\n]", line) if p != ""]
                if len(parts) < 2:
                    continue
                params[parts[0].lower()] = np.float32(parts[1])
        for k, v in params.items():
            setattr(self, k, v)
        for k in ("rotview", "nu", "nv", "nx", "ny", "nz"):
            setattr(self, k, int(getattr(self, k)))
        self.off_a = -self.off_a
        self.da = self.du / self.dsd
        self.UpdateAngularSampling()

    def UpdateAngularSampling(self):
        self.angles = (np.arange(0, self.rotview, dtype=np.float32) * 2 * np.pi / self.rotview).tolist()

    def get_det_sz(self, type_projector=0):
        return [self.da, self.dv]

    def get_det_off(self, type_projector=0):
        return [self.off_a, self.off_v]

    def get_img_shape(self):
        return [self.nx, self.ny, self.nz]

    def get_sino_shape(self):
        return [self.nu, self.rotview, self.nv]

    def cSetDevice(self, device):
        return N.lib.SetDevice(int(device))

    # ---- ramp filter (Filter.cu:432 / :476) ----
    def cFilter4d(self, sino, type_filter=0, type_projector=0):
        sino = np.ascontiguousarray(sino, np.float32)
        fsino = np.zeros(sino.shape, np.float32)
        N.lib.cFilterFanFilter(_fptr(fsino), _fptr(sino), sino.shape[0], sino.shape[4], sino.shape[1],
                               sino.shape[2], sino.shape[3], self.da, self.dv, self.off_a, self.off_v,
                               self.dsd, self.dso, int(type_filter), int(type_projector))
        N.check_last()
        return fsino

    def cFilter3d(self, sino, type_filter=0, type_projector=0):
        return self.cFilter4d(sino[..., np.newaxis, :], type_filter, type_projector)[..., 0, :]

    def cFilterParallel4d(self, sino, type_filter=0):
        sino = np.ascontiguousarray(sino, np.float32)
        fsino = np.zeros(sino.shape, np.float32)
        N.lib.cFilterParallelFilter(_fptr(fsino), _fptr(sino), sino.shape[0], sino.shape[4], sino.shape[1],
                                    sino.shape[2], sino.shape[3], self.da, self.dv, self.off_a, self.off_v,
                                    self.dsd, self.dso, int(type_filter), 0)
        N.check_last()
        return fsino

    # ---- DD fan projector (DistanceDriven.cu:386 / :793) ----
    def _angles(self, angles):
        if angles is None:
            return np.array(self.angles, np.float32)
        return np.ascontiguousarray(angles, np.float32)

    def _fan_args(self, img_shape5, sino_shape5, type_projector):
        B, nx, ny, nz, C = img_shape5
        _, nu, nview, nv, _ = sino_shape5
        return (B, C, nx, ny, nz, self.dx, self.dy, self.dz, nu, nview, nv, self.da, self.dv, self.off_a,
                self.off_v, self.dsd, self.dso, int(type_projector))

    def cDDFanProjection4d(self, img, angles=None, sino_shape=None, type_projector=0):
        img = np.ascontiguousarray(img, np.float32)
        angles = self._angles(angles)
        if sino_shape is None:
            sino_shape = [self.nu, len(angles), self.nv]
        sino = _out([img.shape[0], sino_shape[0], sino_shape[1], sino_shape[2], img.shape[4]], np.float32)
        N.lib.cDistanceDrivenFanProjection(_fptr(sino), _fptr(img), _fptr(angles),
                                           *self._fan_args(img.shape, sino.shape, type_projector))
        N.check_last()
        return sino

    def cDDFanProjection3d(self, img, angles=None, sino_shape=None, type_projector=0):
        angles = self._angles(angles)
        if sino_shape is None:
            sino_shape = [self.nu, len(angles), 1]
        sino = self.cDDFanProjection4d(img[..., np.newaxis, :], angles, sino_shape, type_projector)
        return np.squeeze(sino, -2)

    def cDDFanBackprojection4d(self, sino, angles=None, img_shape=None, type_projector=0):
        sino = np.ascontiguousarray(sino, np.float32)
        angles = self._angles(angles)
        if img_shape is None:
            img_shape = [self.nx, self.ny, self.nz]
        img = _out([sino.shape[0], img_shape[0], img_shape[1], img_shape[2], sino.shape[4]], np.float32)
        N.lib.cDistanceDrivenFanBackprojection(_fptr(img), _fptr(sino), _fptr(angles),
                                               *self._fan_args(img.shape, sino.shape, type_projector))
        N.check_last()
        return img

    def cDDFanBackprojection3d(self, sino, angles=None, img_shape=None, type_projector=0):
        if img_shape is None:
            img_shape = [self.nx, self.ny, 1]
        img = self.cDDFanBackprojection4d(sino[..., np.newaxis, :], angles, img_shape, type_projector)
        return img[..., 0, :]

    # ---- pixel-driven FBP backprojection (python/ReconNet_no_tf.py:101-131) ----
    def cPixelBackprojection4d(self, sino, angles=None, img_shape=None, type_projector=0):
        sino = np.ascontiguousarray(sino, np.float32)
        angles = self._angles(angles)
        if img_shape is None:
            img_shape = [self.nx, self.ny, self.nz]
        img = _out([sino.shape[0], img_shape[0], img_shape[1], img_shape[2], sino.shape[4]], np.float32)
        N.lib.cPixelDrivenFanBackprojection(_fptr(img), _fptr(sino), _fptr(angles),
                                            *self._fan_args(img.shape, sino.shape, type_projector))
        N.check_last()
        return img

    def cPixelBackprojection3d(self, sino, angles=None, img_shape=None, type_projector=0):
        if img_shape is None:
            img_shape = [self.nx, self.ny, 1]
        img = self.cPixelBackprojection4d(sino[..., np.newaxis, :], angles, img_shape, type_projector)
        return img[..., 0, :]

    # ---- Siddon fan pair (python/ReconNet_no_tf.py:290-394) ----
    def cSiddonFanProjection4d(self, img, angles=None, sino_shape=None, type_projector=0):
        img = np.ascontiguousarray(img, np.float32)
        angles = self._angles(angles)
        if sino_shape is None:
            sino_shape = [self.nu, len(angles), self.nv]
        sino = _out([img.shape[0], sino_shape[0], sino_shape[1], sino_shape[2], img.shape[4]], np.float32)
        N.lib.cSiddonFanProjection(_fptr(sino), _fptr(img), _fptr(angles),
                                   *self._fan_args(img.shape, sino.shape, type_projector))
        N.check_last()
        return sino

    def cSiddonFanProjection3d(self, img, angles=None, sino_shape=None, type_projector=0):
        angles = self._angles(angles)
        if sino_shape is None:
            sino_shape = [self.nu, len(angles), 1]
        sino = self.cSiddonFanProjection4d(img[..., np.newaxis, :], angles, sino_shape, type_projector)
        return np.squeeze(sino, -2)

    def cSiddonFanBackprojection4d(self, sino, angles=None, img_shape=None, type_projector=0):
        sino = np.ascontiguousarray(sino, np.float32)
        angles = self._angles(angles)
        if img_shape is None:
            img_shape = [self.nx, self.ny, self.nz]
        img = _out([sino.shape[0], img_shape[0], img_shape[1], img_shape[2], sino.shape[4]], np.float32)
        N.lib.cSiddonFanBackprojection(_fptr(img), _fptr(sino), _fptr(angles),
                                       *self._fan_args(img.shape, sino.shape, type_projector))
        N.check_last()
        return img

    def cSiddonFanBackprojection3d(self, sino, angles=None, img_shape=None, type_projector=0):
        if img_shape is None:
            img_shape = [self.nx, self.ny, 1]
        img = self.cSiddonFanBackprojection4d(sino[..., np.newaxis, :], angles, img_shape, type_projector)
        return img[..., 0, :]

    def cSiddonFanNormImg4d(self, sino, wsino=None, angles=None, img_shape=None, type_projector=0):
        """normImg = BP(W * FP(1)) with the Siddon pair (ReconNet_no_tf.py:359-380)."""
        angles = self._angles(angles)
        wsino = np.ones(sino.shape, np.float32) if wsino is None else np.asarray(wsino, np.float32)
        if img_shape is None:
            img_shape = [self.nx, self.ny, self.nz]
        ones = np.ones([sino.shape[0], img_shape[0], img_shape[1], img_shape[2], sino.shape[4]], np.float32)
        fp = self.cSiddonFanProjection4d(ones, angles, list(sino.shape[1:4]), type_projector)
        return self.cSiddonFanBackprojection4d(fp * wsino, angles, img_shape, type_projector)

    def cSiddonFanNormImg3d(self, sino, wsino=None, angles=None, img_shape=None, type_projector=0):
        if img_shape is None:
            img_shape = [self.nx, self.ny, 1]
        w = None if wsino is None else np.asarray(wsino)[..., np.newaxis, :]
        norm = self.cSiddonFanNormImg4d(np.asarray(sino)[..., np.newaxis, :], w, angles, img_shape, type_projector)
        return norm[..., 0, :]

    def cDDFanNormImg4d(self, sino, wsino=None, angles=None, img_shape=None, type_projector=0):
        """normImg = BP(W * FP(1)) (ReconNet_no_tf.py:202-223)."""
        angles = self._angles(angles)
        wsino = np.ones(sino.shape, np.float32) if wsino is None else np.asarray(wsino, np.float32)
        if img_shape is None:
            img_shape = [self.nx, self.ny, self.nz]
        ones = np.ones([sino.shape[0], img_shape[0], img_shape[1], img_shape[2], sino.shape[4]], np.float32)
        fp = self.cDDFanProjection4d(ones, angles, sino.shape[1:4], type_projector)
        return self.cDDFanBackprojection4d(fp * wsino, angles, img_shape, type_projector)

    def cDDFanNormImg3d(self, sino, wsino=None, angles=None, img_shape=None, type_projector=0):
        wsino = np.ones(sino.shape, np.float32) if wsino is None else np.asarray(wsino, np.float32)
        if img_shape is None:
            img_shape = [self.nx, self.ny, 1]
        n = self.cDDFanNormImg4d(sino[..., np.newaxis, :], wsino[..., np.newaxis, :], angles, img_shape,
                                 type_projector)
        return n[..., 0, :]

    # ---- OS-SQS (ossqs.cu:12 semantics) ----
    def cSiddonFanOSSQS4d(self, nSubsets, img, sino, normImg, wsino=None, angles=None, order=None, lb=None,
                          ub=None, type_projector=0, lam=1):
        """cOSSQS with the Siddon pair, as ReconNet_no_tf.py:396-440."""
        return self._ossqs(N.lib.cOSSQS, nSubsets, img, sino, normImg, wsino, angles, order, lb, ub,
                           type_projector, lam)

    def cSiddonFanOSSQS3d(self, nSubsets, img, sino, normImg, wsino=None, angles=None, order=None, lb=None,
                          ub=None, type_projector=0, lam=1):
        wsino = np.ones(sino.shape, np.float32) if wsino is None else np.asarray(wsino, np.float32)
        res = self.cSiddonFanOSSQS4d(nSubsets, img[..., np.newaxis, :], sino[..., np.newaxis, :],
                                     normImg[..., np.newaxis, :], wsino[..., np.newaxis, :], angles, order, lb, ub,
                                     type_projector, lam)
        return res[..., 0, :]

    def cDDFanOSSQS4d(self, nSubsets, img, sino, normImg, wsino=None, angles=None, order=None, lb=None, ub=None,
                      type_projector=0, lam=1):
        """Same arguments as cSiddonFanOSSQS4d with the DD pair (cDDFanOSSQS)."""
        return self._ossqs(N.lib.cDDFanOSSQS, nSubsets, img, sino, normImg, wsino, angles, order, lb, ub,
                           type_projector, lam)

    def _ossqs(self, fn, nSubsets, img, sino, normImg, wsino, angles, order, lb, ub, type_projector, lam):
        img = np.ascontiguousarray(img, np.float32)
        sino = np.asarray(sino, np.float32)
        normImg = np.ascontiguousarray(normImg, np.float32)
        lb = np.finfo(np.float32).min if lb is None else lb
        ub = np.finfo(np.float32).max if ub is None else ub
        wsino = np.ones(sino.shape, np.float32) if wsino is None else np.asarray(wsino, np.float32)
        angles = self._angles(angles)
        nviewPerSubset = int(np.ceil(sino.shape[2] / float(nSubsets)))
        if order is not None:
            angles = np.ascontiguousarray(angles[order])
            sino = sino[..., order, :, :]
            wsino = wsino[..., order, :, :]
        sino = np.ascontiguousarray(sino, np.float32)
        wsino = np.ascontiguousarray(wsino, np.float32)
        res = np.zeros(img.shape, np.float32)
        B, nx, ny, nz, C = img.shape
        fn(_fptr(res), _fptr(img), _fptr(sino), _fptr(normImg), _fptr(wsino), _fptr(angles), float(lb), float(ub),
           nviewPerSubset, int(nSubsets), B, C, nx, ny, nz, self.dx, self.dy, self.dz, sino.shape[1],
           sino.shape[2], sino.shape[3], self.da, self.dv, self.off_a, self.off_v, self.dsd, self.dso,
           int(type_projector), float(lam))
        N.check_last()
        return res

    def cDDFanOSSQS3d(self, nSubsets, img, sino, normImg, wsino=None, angles=None, order=None, lb=None, ub=None,
                      type_projector=0, lam=1):
        wsino = np.ones(sino.shape, np.float32) if wsino is None else np.asarray(wsino, np.float32)
        res = self.cDDFanOSSQS4d(nSubsets, img[..., np.newaxis, :], sino[..., np.newaxis, :],
                                 normImg[..., np.newaxis, :], wsino[..., np.newaxis, :], angles, order, lb, ub,
                                 type_projector, lam)
        return res[..., 0, :]

    # ---- tomosynthesis DD (DistanceDriven3D.cu:346 / :666) ----
    def _tomo_args(self, img_shape5, prj_shape5):
        B, nx, ny, nz, C = img_shape5
        _, nu, nview, nv, _ = prj_shape5
        return (B, C, nx, ny, nz, self.dx, self.dy, self.dz, self.cx, self.cy, self.cz, nu, nview, nv, self.du,
                self.dv, self.off_u, self.off_v)

    def cDDTomoProjection4d(self, img, detCenter, src):
        img = np.ascontiguousarray(img, np.float32)
        detCenter = np.ascontiguousarray(detCenter, np.float32)
        src = np.ascontiguousarray(src, np.float32)
        prj = _out([img.shape[0], self.nu, detCenter.shape[0], self.nv, img.shape[-1]], np.float32)
        N.lib.cDistanceDrivenTomoProjection(_fptr(prj), _fptr(img), _fptr(detCenter), _fptr(src),
                                            *self._tomo_args(img.shape, prj.shape))
        N.check_last()
        return prj

    def cDDTomoBackprojection4d(self, prj, detCenter, src):
        prj = np.ascontiguousarray(prj, np.float32)
        detCenter = np.ascontiguousarray(detCenter, np.float32)
        src = np.ascontiguousarray(src, np.float32)
        img = _out([prj.shape[0], self.nx, self.ny, self.nz, prj.shape[-1]], np.float32)
        N.lib.cDistanceDrivenTomoBackprojection(_fptr(img), _fptr(prj), _fptr(detCenter), _fptr(src),
                                                *self._tomo_args(img.shape, prj.shape))
        N.check_last()
        return img

    def cDDTomoNormImg4d(self, prj, detCenter, src, mask=None):
        img = np.ones([prj.shape[0], self.nx, self.ny, self.nz, prj.shape[-1]], np.float32)
        if mask is None:
            mask = np.ones_like(img)
        fp = self.cDDTomoProjection4d(img * mask, detCenter, src)
        return self.cDDTomoBackprojection4d(fp, detCenter, src) * mask

    # ---- Siddon cone pair, arbitrary geometry (python/ReconNet_no_tf.py:503-610) ----
    def cSiddonConeProjectionAbitrary4d(self, img, detCenter, detU, detV, src):
        img = np.ascontiguousarray(img, np.float32)
        geo = [np.ascontiguousarray(a, np.float32) for a in (detCenter, detU, detV, src)]
        prj = np.zeros([img.shape[0], self.nu, geo[0].shape[0], self.nv, img.shape[-1]], np.float32)
        N.lib.cSiddonConeProjectionAbitrary(_fptr(prj), _fptr(img), *[_fptr(a) for a in geo],
                                            *self._tomo_args(img.shape, prj.shape))
        N.check_last()
        return prj

    def cSiddonConeBackprojectionAbitrary4d(self, prj, detCenter, detU, detV, src):
        prj = np.ascontiguousarray(prj, np.float32)
        geo = [np.ascontiguousarray(a, np.float32) for a in (detCenter, detU, detV, src)]
        img = np.zeros([prj.shape[0], self.nx, self.ny, self.nz, prj.shape[-1]], np.float32)
        N.lib.cSiddonConeBackprojectionAbitrary(_fptr(img), _fptr(prj), *[_fptr(a) for a in geo],
                                                *self._tomo_args(img.shape, prj.shape))
        N.check_last()
        return img

    def cSiddonConeNormImgAbitrary4d(self, prj, detCenter, detU, detV, src, mask=None):
        img = np.ones([prj.shape[0], self.nx, self.ny, self.nz, prj.shape[-1]], np.float32)
        if mask is None:
            mask = np.ones_like(img)
        fp = self.cSiddonConeProjectionAbitrary4d(img * mask, detCenter, detU, detV, src)
        return self.cSiddonConeBackprojectionAbitrary4d(fp, detCenter, detU, detV, src) * mask

    def cSiddonConeAbitraryOSSQS4d(self, nSubsets, img, prj, normImg, detCenter, detU, detV, src, mask=None,
                                   order=None, lb=None, ub=None, lam=1):
        img = np.ascontiguousarray(img, np.float32)
        prj = np.asarray(prj, np.float32)
        normImg = np.ascontiguousarray(normImg, np.float32)
        geo = [np.asarray(a, np.float32) for a in (detCenter, detU, detV, src)]
        mask = np.ones(img.shape, np.float32) if mask is None else np.ascontiguousarray(mask, np.float32)
        nviewPerSubset = int(np.ceil(prj.shape[2] / float(nSubsets)))
        lb = np.finfo(np.float32).min if lb is None else lb
        ub = np.finfo(np.float32).max if ub is None else ub
        if order is not None:
            prj = prj[:, :, order, :, :]
            geo = [a[order, ...] for a in geo]
        prj = np.ascontiguousarray(prj, np.float32)
        geo = [np.ascontiguousarray(a, np.float32) for a in geo]
        res = np.zeros(img.shape, np.float32)
        B, nx, ny, nz, C = img.shape
        N.lib.cOSSQSConeAbitrary(_fptr(res), _fptr(img), _fptr(prj), _fptr(normImg), _fptr(mask),
                                 *[_fptr(a) for a in geo], float(lb), float(ub), nviewPerSubset, int(nSubsets),
                                 *self._tomo_args(img.shape, prj.shape), 2, float(lam))
        N.check_last()
        return res

    # ---- TV surrogate (TotalVariation.cu:70) ----
    def cTVSQS2d(self, img):
        img = np.ascontiguousarray(img, np.float32)
        if img.ndim != 4 or img.shape[0] != 1 or img.shape[-1] != 1:
            raise ValueError("img.shape must be [1, _, _, 1]")
        grad = np.zeros(img.shape, np.float32)
        norm = np.zeros(img.shape, np.float32)
        tv = N.lib.cTVSQS2D(_fptr(grad), _fptr(norm), _fptr(img), img.shape[1], img.shape[2])
        N.check_last()
        return grad, norm, tv


def _shortscan(reconNet, kind, sigma=30.0, theta=10 * np.pi / 180, riess_mask=0):
    ang = np.ascontiguousarray(np.asarray(reconNet.angles, np.float32).ravel())
    nu, nview = int(reconNet.nu), int(ang.size)
    w = np.zeros((nu, nview), np.float32)
    N.check(N.lib.rn_fan_shortscan_weights_host(_fptr(w), _fptr(ang), nu, nview, float(reconNet.da),
                                                float(reconNet.off_a), int(kind), float(sigma), float(theta),
                                                int(riess_mask)))
    return w[None, :, :, None]


def ParkerWeighting(reconNet):
    """Parker short-scan weights for reconNet.angles over [0, pi + 2 gamma],
    shape [1, nu, nview, 1] -- the reference's ParkerWeighting
    (python/ReconNet_no_tf.py:640-659), computed on the GPU by
    rn_fan_shortscan_weights_host (kernel in csrc/shortscan.cu)."""
    return _shortscan(reconNet, N.RN_WEIGHT_PARKER)


def RiessWeighting(reconNet, sigma=30, theta=10 * np.pi / 180, whole_view_exception=False):
    """Riess short-scan weights, shape [1, nu, nview, 1] -- the reference's
    RiessWeighting (python/ReconNet_no_tf.py:665-693) on the GPU.  By default
    the views with theta < beta < pi + 2 gamma - theta keep only channel 0
    unsmoothed, which is what the reference's np.where(np.all(...)) selects;
    whole_view_exception=True keeps those whole views unsmoothed instead."""
    return _shortscan(reconNet, N.RN_WEIGHT_RIESS, sigma, theta, 1 if whole_view_exception else 0)
