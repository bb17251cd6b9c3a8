"""PyTorch-facing device API: plans over CUDA tensors and autograd.

``FanPlan`` owns a native ``rn_fan_plan`` (geometry tables + scratch) and runs
the sm_100a kernels on the caller's current CUDA stream with the tensors'
device pointers.  ``FanProjectFn`` mirrors the reference's TF op + registered
gradient pair (ReconNet4D/zOpsReconNet.cc:26-82, python/ReconNet.py:773-800):
forward = DD forward projection, backward = the matched (exact-transpose)
backprojection.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import Optional, Sequence, Tuple

import numpy as np
import torch

from . import _native as N
from .geometry import CylGeometry, FanGeometry  # noqa: F401  (re-exported)


def _stream_ptr(device: torch.device) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def _dev_ptr(t: torch.Tensor) -> int:
    if not t.is_cuda:
        raise ValueError("reconnet_b200 device API needs CUDA tensors")
    if t.dtype != torch.float32 or not t.is_contiguous():
        raise ValueError("tensors must be contiguous float32")
    return t.data_ptr()


class FanPlan:
    """Native plan for a batch of fan-beam problems.

    Reference layout (``nview_per_slice`` is None): image ``[B, nx, ny, nz, C]``,
    sinogram ``[B, nu, nview, nv, C]``, one angle list.

    Ragged layout: ``nbatches`` independent ``[nx, ny]`` slices; slice ``s`` has
    ``nview_per_slice[s]`` views; the sinogram is packed as the concatenation
    of per-slice ``[nu, nview_s]`` blocks (a flat tensor)."""

    def __init__(self, geom: FanGeometry, angles, nbatches: int = 1, nchannels: int = 1,
                 nview_per_slice: Optional[Sequence[int]] = None, device=None):
        self.geom = geom
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.angles = np.ascontiguousarray(np.asarray(angles, np.float32).ravel())
        self.nbatches, self.nchannels = int(nbatches), int(nchannels)
        self.ragged = nview_per_slice is not None
        self._plan = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            st = _stream_ptr(self.device)
            aptr = self.angles.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
            if self.ragged:
                nvs = np.ascontiguousarray(np.asarray(nview_per_slice, np.int32))
                if nvs.sum() != self.angles.size:
                    raise ValueError("angles must hold sum(nview_per_slice) entries")
                self.nview_per_slice = nvs
                g = geom.native(self.nbatches, 1, int(nvs.sum()))
                g.nz = g.nv = 1
                N.check(N.lib.rn_fan_plan_create_ragged(ctypes.byref(self._plan), ctypes.byref(g),
                                                        nvs.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), aptr, st))
                self.img_shape = (self.nbatches, geom.nx, geom.ny)
                self.sino_shape = (int(nvs.sum()) * geom.nu,)
            else:
                self.nview = self.angles.size
                g = geom.native(self.nbatches, self.nchannels, self.nview)
                N.check(N.lib.rn_fan_plan_create(ctypes.byref(self._plan), ctypes.byref(g), aptr, st))
                self.img_shape = (self.nbatches, geom.nx, geom.ny, geom.nz, self.nchannels)
                self.sino_shape = (self.nbatches, geom.nu, self.nview, geom.nv, self.nchannels)
        self.total_views = int(N.lib.rn_fan_plan_total_views(self._plan))

    def __del__(self):
        p = getattr(self, "_plan", None)
        if p is not None and p.value:
            try:
                N.lib.rn_fan_plan_destroy(p)
            except Exception:
                pass
            self._plan = ctypes.c_void_p()

    # updates per call, the unit of the Gray/s metric: ray-line (FP) and
    # pixel-view (BP) footprint integrations
    def fp_updates(self) -> int:
        g = self.geom
        if self.ragged:
            return int(self.total_views) * g.nu * g.ny
        return self.nbatches * self.nchannels * g.nv * self.nview * g.nu * g.ny

    def bp_updates(self) -> int:
        g = self.geom
        if self.ragged:
            return int(self.total_views) * g.nx * g.ny
        return self.nbatches * self.nchannels * g.nz * self.nview * g.nx * g.ny

    def project(self, img: torch.Tensor, out: Optional[torch.Tensor] = None, siddon: bool = False) -> torch.Tensor:
        """Distance-driven forward projection, or the Siddon ray-length
        projection with ``siddon=True`` (its transpose: ``backproject(...,
        N.RN_TYPE_SIDDON)``)."""
        if tuple(img.shape) != self.img_shape:
            raise ValueError(f"image shape {tuple(img.shape)} != {self.img_shape}")
        if out is None:
            out = torch.empty(self.sino_shape, dtype=torch.float32, device=img.device)
        fn = N.lib.rn_fan_project_siddon if siddon else N.lib.rn_fan_project
        N.check(fn(self._plan, _dev_ptr(out), _dev_ptr(img), _stream_ptr(img.device)))
        return out

    def backproject(self, sino: torch.Tensor, type_projector: int = N.RN_TYPE_MATCHED,
                    out: Optional[torch.Tensor] = None, accumulate: bool = False) -> torch.Tensor:
        if tuple(sino.shape) != self.sino_shape:
            raise ValueError(f"sinogram shape {tuple(sino.shape)} != {self.sino_shape}")
        if out is None:
            out = torch.empty(self.img_shape, dtype=torch.float32, device=sino.device)
        N.check(N.lib.rn_fan_backproject(self._plan, _dev_ptr(out), _dev_ptr(sino), int(type_projector),
                                         int(bool(accumulate)), _stream_ptr(sino.device)))
        return out

    KERNEL_KINDS = ("lines", "fp", "tables", "bp", "other")

    def set_timing(self, enable: bool) -> None:
        """Bracket every kernel launch with CUDA events (for per-kernel timing)."""
        N.check(N.lib.rn_fan_plan_set_timing(self._plan, int(bool(enable))))

    def read_timing(self):
        """-> ({kind: (total_ms, launches)}, total kernels launched by this plan)."""
        n = len(self.KERNEL_KINDS)
        ms = (ctypes.c_float * n)()
        cnt = (ctypes.c_int * n)()
        launches = ctypes.c_longlong()
        N.check(N.lib.rn_fan_plan_read_timing(self._plan, ms, cnt, n, ctypes.byref(launches)))
        return {k: (float(ms[i]), int(cnt[i])) for i, k in enumerate(self.KERNEL_KINDS)}, int(launches.value)

    def launches(self) -> int:
        """Total number of kernels this plan has launched."""
        launches = ctypes.c_longlong()
        N.check(N.lib.rn_fan_plan_read_timing(self._plan, None, None, 0, ctypes.byref(launches)))
        return launches.value

    def check(self) -> None:
        """Synchronise and raise if a device-side bounded wait gave up."""
        N.check(N.lib.rn_fan_plan_check(self._plan, _stream_ptr(self.device)))

    def set_spin_limit(self, polls: int = -1) -> None:
        """Polls each device-side chunk wait makes before giving up (-1: the default)."""
        N.check(N.lib.rn_fan_plan_set_spin_limit(self._plan, int(polls)))

    def autotune(self, img: torch.Tensor, type_projector: int = N.RN_TYPE_MATCHED,
                 sino: Optional[torch.Tensor] = None) -> Tuple[int, int, int]:
        """Time the launch-parameter candidates of this plan's forward
        projection (Siddon for ``N.RN_TYPE_SIDDON``) and backprojection of
        ``type_projector`` on ``img`` and keep the fastest (cached per
        geometry for the process).  ``sino`` (overwritten) is scratch.
        Returns (fp_views, fp_lines, bp_parts)."""
        if tuple(img.shape) != self.img_shape:
            raise ValueError(f"image shape {tuple(img.shape)} != {self.img_shape}")
        if sino is None:
            sino = torch.empty(self.sino_shape, dtype=torch.float32, device=img.device)
        N.check(N.lib.rn_fan_plan_autotune(self._plan, _dev_ptr(sino), _dev_ptr(img), int(type_projector),
                                           _stream_ptr(img.device)))
        return self.tuning()

    def tuning(self) -> Tuple[int, int, int]:
        """(fp_views, fp_lines, bp_parts) in use; bp_parts 0 = built-in."""
        v, r, b = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        N.check(N.lib.rn_fan_plan_get_tuning(self._plan, ctypes.byref(v), ctypes.byref(r), ctypes.byref(b)))
        return v.value, r.value, b.value

    def set_tuning(self, fp_views: int = 0, fp_lines: int = 0, bp_parts: int = 0) -> None:
        """Set the launch parameters (0 = built-in choice) on the current stream."""
        N.check(N.lib.rn_fan_plan_set_tuning(self._plan, int(fp_views), int(fp_lines), int(bp_parts),
                                             _stream_ptr(self.device)))

    def sqs_update(self, x_out, x_in, prj_s, w_s, norm_img, lam=1.0, beta=0.0, n_subsets=1,
                   lb=None, ub=None, type_projector=N.RN_TYPE_MATCHED):
        """One OS-SQS subset step on every slice (this plan = the subset's views)."""
        lb = float(np.finfo(np.float32).min) if lb is None else float(lb)
        ub = float(np.finfo(np.float32).max) if ub is None else float(ub)
        N.check(N.lib.rn_fan_sqs_update(self._plan, _dev_ptr(x_out), _dev_ptr(x_in), _dev_ptr(prj_s),
                                        _dev_ptr(w_s), _dev_ptr(norm_img), float(lam), float(beta),
                                        int(n_subsets), lb, ub, int(type_projector),
                                        _stream_ptr(x_in.device)))
        return x_out


class StreamedFanPair:
    """Forward projection followed by the backprojection of its result for a
    ragged batch of independent slices held in pinned host memory, with the
    transfers overlapped.

    The slices run in ``groups`` contiguous groups, each with its own plan, and
    the device buffers are double-buffered across calls.  One group gives the
    best throughput over a sequence of calls (no extra launch tails); more
    groups also overlap the copies within a single call.  A group's
    host-to-device copy runs on one copy stream, its FP + BP on the caller's
    current stream, and its device-to-host copy on a second copy stream.  So a
    call's copies overlap the computation of its other groups and of the
    neighbouring calls (the next call's inputs are copied while this call
    computes).  Results are identical to one plan over the whole batch: every
    slice is processed independently."""

    def __init__(self, geom: FanGeometry, angles, nview_per_slice: Sequence[int], groups: int = 1,
                 type_projector: int = N.RN_TYPE_MATCHED, device=None):
        from types import SimpleNamespace
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        counts = np.asarray(nview_per_slice, np.int64)
        angles = np.asarray(angles, np.float32).ravel()
        if counts.sum() != angles.size:
            raise ValueError("angles must hold sum(nview_per_slice) entries")
        nsl = len(counts)
        ngroups = max(1, min(int(groups), nsl))
        bounds = np.linspace(0, nsl, ngroups + 1).round().astype(int)
        offs = np.concatenate([[0], np.cumsum(counts)])
        self.type_projector = int(type_projector)
        self.nslices = nsl
        self.groups = []
        for g in range(ngroups):
            s0, s1 = int(bounds[g]), int(bounds[g + 1])
            plan = FanPlan(geom, angles[offs[s0]:offs[s1]], nbatches=s1 - s0, nview_per_slice=counts[s0:s1],
                           device=self.device)
            bufs = [SimpleNamespace(x=torch.empty(plan.img_shape, device=self.device),
                                    b=torch.empty(plan.img_shape, device=self.device),
                                    h2d=torch.cuda.Event(), comp=torch.cuda.Event(), d2h=torch.cuda.Event())
                    for _ in range(2)]
            self.groups.append(SimpleNamespace(s0=s0, s1=s1, plan=plan, bufs=bufs,
                                               p=torch.empty(plan.sino_shape, device=self.device)))
        self.h2d_stream = torch.cuda.Stream(self.device)
        self.d2h_stream = torch.cuda.Stream(self.device)
        self.done = torch.cuda.Event()
        self.inputs_read = torch.cuda.Event()
        self.calls = 0

    def updates(self) -> int:
        return sum(g.plan.fp_updates() + g.plan.bp_updates() for g in self.groups)

    def __call__(self, host_img: torch.Tensor, host_out: torch.Tensor) -> torch.cuda.Event:
        """host_img, host_out: pinned float32 [S, nx, ny] host tensors.  Enqueues
        the work and returns an event that completes when host_out is written.
        The copies are asynchronous: host_img may be overwritten only after
        ``self.inputs_read`` (recorded after this call's host-to-device copies)
        or the returned event has completed, and host_out read only after the
        returned event has."""
        if host_img.shape[0] != self.nslices or host_out.shape[0] != self.nslices:
            raise ValueError("host tensors must hold one [nx, ny] image per slice")
        comp = torch.cuda.current_stream(self.device)
        k = self.calls & 1
        self.calls += 1
        for g in self.groups:
            bf = g.bufs[k]
            self.h2d_stream.wait_event(bf.comp)         # the FP two calls ago has read bf.x
            with torch.cuda.stream(self.h2d_stream):
                bf.x.copy_(host_img[g.s0:g.s1], non_blocking=True)
                bf.h2d.record(self.h2d_stream)
            comp.wait_event(bf.h2d)
            comp.wait_event(bf.d2h)                     # the copy of bf.b two calls ago is done
            g.plan.project(bf.x, out=g.p)
            g.plan.backproject(g.p, self.type_projector, out=bf.b)
            bf.comp.record(comp)
            self.d2h_stream.wait_event(bf.comp)
            with torch.cuda.stream(self.d2h_stream):
                host_out[g.s0:g.s1].copy_(bf.b, non_blocking=True)
                bf.d2h.record(self.d2h_stream)
        self.inputs_read.record(self.h2d_stream)
        self.done.record(self.d2h_stream)
        return self.done

    def check(self) -> None:
        for g in self.groups:
            g.plan.check()


class FanProjectFn(torch.autograd.Function):
    """y = A x with dL/dx = B dL/dy, B the backprojection of type `grad_type`:
    the matched transpose A^T by default (the exact gradient), or the
    reference's iterative backprojection (type 0), which is how the
    reference registers the gradient of its projection op
    (python/ReconNet.py:773-800)."""

    @staticmethod
    def forward(ctx, img, plan: FanPlan, grad_type: int = N.RN_TYPE_MATCHED):
        ctx.plan = plan
        ctx.grad_type = grad_type
        return plan.project(img.contiguous())

    @staticmethod
    def backward(ctx, gy):
        return ctx.plan.backproject(gy.contiguous(), ctx.grad_type), None, None


class FanBackprojectFn(torch.autograd.Function):
    """x = B y (backprojection of type `bp_type`, matched by default) with
    dL/dy = A dL/dx (python/ReconNet.py:801-830 registers the projection as
    the backprojection's gradient)."""

    @staticmethod
    def forward(ctx, sino, plan: FanPlan, bp_type: int = N.RN_TYPE_MATCHED):
        ctx.plan = plan
        return plan.backproject(sino.contiguous(), bp_type)

    @staticmethod
    def backward(ctx, gx):
        return ctx.plan.project(gx.contiguous()), None, None


def fan_project(img: torch.Tensor, plan: FanPlan, grad_type: int = N.RN_TYPE_MATCHED) -> torch.Tensor:
    return FanProjectFn.apply(img, plan, grad_type)


def fan_backproject(sino: torch.Tensor, plan: FanPlan, bp_type: int = N.RN_TYPE_MATCHED) -> torch.Tensor:
    return FanBackprojectFn.apply(sino, plan, bp_type)


def filter_sino(sino: torch.Tensor, geom: FanGeometry, type_filter: int = 0, fan: bool = True) -> torch.Tensor:
    """Ramp filter (cFilterFan::Filter, Filter.cu:216) on a [B, nu, nview, nv, C] CUDA tensor."""
    out = torch.empty_like(sino)
    B, nu, nview, nv, C = sino.shape
    N.check(N.lib.rn_filter(_dev_ptr(out), _dev_ptr(sino), B, C, nu, nview, nv, float(geom.da),
                            float(geom.off_a), float(geom.dsd), float(geom.dso), int(type_filter), int(bool(fan)),
                            _stream_ptr(sino.device)))
    return out


@dataclass
class ConeGeometry:
    """Cone-beam grid and detector (the SiddonCone setup, SiddonCone.cu:126-201):
    grid of nx x ny x nz voxels (dx, dy, dz mm) centred at (cx, cy, cz);
    detector of nu x nv cells (du, dv mm) with offsets off_u, off_v in cells."""
    nx: int = 512
    ny: int = 512
    nz: int = 128
    dx: float = 0.8
    dy: float = 0.8
    dz: float = 1.0
    cx: float = 0.0
    cy: float = 0.0
    cz: float = 0.0
    nu: int = 736
    nv: int = 736
    du: float = 0.6
    dv: float = 0.6
    off_u: float = 0.0
    off_v: float = 0.0

    def native(self, nbatches: int, nchannels: int, nview: int) -> N.RnConeGeom:
        g = N.RnConeGeom()
        g.nBatches, g.nChannels = nbatches, nchannels
        g.nx, g.ny, g.nz = self.nx, self.ny, self.nz
        g.dx, g.dy, g.dz, g.cx, g.cy, g.cz = self.dx, self.dy, self.dz, self.cx, self.cy, self.cz
        g.nu, g.nview, g.nv = self.nu, nview, self.nv
        g.du, g.dv, g.off_u, g.off_v = self.du, self.dv, self.off_u, self.off_v
        return g


class ConePlan:
    """Siddon cone-beam pair with arbitrary per-view geometry on CUDA tensors:
    image ``[B, nx, ny, nz, C]``, projections ``[B, nu, nview, nv, C]``;
    ``det_center``, ``det_u``, ``det_v``, ``src`` are ``[nview, 3]`` (mm).
    ``project`` traces ray lengths (SiddonCone.cu:20-42), ``backproject`` is
    its exact transpose."""

    def __init__(self, geom: ConeGeometry, det_center, det_u, det_v, src, nbatches: int = 1, nchannels: int = 1,
                 device=None):
        self.geom = geom
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        geo = [np.ascontiguousarray(np.asarray(a, np.float32).reshape(-1, 3)) for a in (det_center, det_u, det_v, src)]
        self.nview = geo[0].shape[0]
        self.nbatches, self.nchannels = int(nbatches), int(nchannels)
        self._plan = ctypes.c_void_p()
        g = geom.native(self.nbatches, self.nchannels, self.nview)
        fp = ctypes.POINTER(ctypes.c_float)
        with torch.cuda.device(self.device):
            N.check(N.lib.rn_cone_plan_create(ctypes.byref(self._plan), ctypes.byref(g),
                                              *[a.ctypes.data_as(fp) for a in geo], _stream_ptr(self.device)))
        self.img_shape = (self.nbatches, geom.nx, geom.ny, geom.nz, self.nchannels)
        self.prj_shape = (self.nbatches, geom.nu, self.nview, geom.nv, self.nchannels)

    def __del__(self):
        p = getattr(self, "_plan", None)
        if p is not None and p.value:
            try:
                N.lib.rn_cone_plan_destroy(p)
            except Exception:
                pass
            self._plan = ctypes.c_void_p()

    def project(self, img: torch.Tensor, out: Optional[torch.Tensor] = None) -> torch.Tensor:
        if tuple(img.shape) != self.img_shape:
            raise ValueError(f"image shape {tuple(img.shape)} != {self.img_shape}")
        if out is None:
            out = torch.empty(self.prj_shape, dtype=torch.float32, device=img.device)
        N.check(N.lib.rn_cone_project(self._plan, _dev_ptr(out), _dev_ptr(img), _stream_ptr(img.device)))
        return out

    def backproject(self, prj: torch.Tensor, out: Optional[torch.Tensor] = None,
                    accumulate: bool = False) -> torch.Tensor:
        if tuple(prj.shape) != self.prj_shape:
            raise ValueError(f"projection shape {tuple(prj.shape)} != {self.prj_shape}")
        if out is None:
            out = torch.empty(self.img_shape, dtype=torch.float32, device=prj.device)
        N.check(N.lib.rn_cone_backproject(self._plan, _dev_ptr(out), _dev_ptr(prj), int(bool(accumulate)),
                                          _stream_ptr(prj.device)))
        return out

    def launches(self) -> int:
        return int(N.lib.rn_cone_plan_launches(self._plan))


def shortscan_weights(angles: torch.Tensor, geom: FanGeometry, kind: str = "parker", sigma: float = 30.0,
                      theta: float = 10 * np.pi / 180, whole_view_exception: bool = False) -> torch.Tensor:
    """Short-scan redundancy weights [nu, nview] on the device for the view
    angles of a float32 CUDA tensor (rn_fan_shortscan_weights): Parker or
    Riess, as the reference's ParkerWeighting / RiessWeighting
    (python/ReconNet_no_tf.py:640-693)."""
    ang = angles.detach().to(torch.float32).contiguous().reshape(-1)
    if not ang.is_cuda:
        raise ValueError("angles must be a CUDA tensor")
    w = torch.empty((geom.nu, ang.numel()), dtype=torch.float32, device=ang.device)
    k = {"parker": N.RN_WEIGHT_PARKER, "riess": N.RN_WEIGHT_RIESS}[kind]
    N.check(N.lib.rn_fan_shortscan_weights(_dev_ptr(w), _dev_ptr(ang), int(geom.nu), int(ang.numel()),
                                           float(geom.da), float(geom.off_a), k, float(sigma), float(theta),
                                           int(bool(whole_view_exception)), _stream_ptr(ang.device)))
    return w


def fbp(sino: torch.Tensor, plan: "FanPlan", geom: FanGeometry, type_filter: int = 0,
        weights: Optional[torch.Tensor] = None, out: Optional[torch.Tensor] = None) -> torch.Tensor:
    """Fan-beam FBP on the device: optional short-scan weights (Parker /
    Riess, [nu, nview] from `shortscan_weights`, or any shape holding nu x
    nview values), multiplied into the sinogram inside the ramp filter's load
    (rn_filter_weighted), then the pixel-driven backprojection with the
    dso^2 / L^2 weight (cPixelDrivenFan) -- the reference's FBP chain
    (ReconNet_no_tf.py:84-131, 640-693).  sino is [B, nu, nview, nv, C] in the
    plan's layout."""
    if weights is None:
        filt = filter_sino(sino, geom, type_filter)
    else:
        B, nu, nview, nv, C = sino.shape
        w = weights.to(device=sino.device, dtype=torch.float32).contiguous()
        if w.numel() != nu * nview:
            raise ValueError(f"weights must hold nu x nview = {nu} x {nview} values, got shape {tuple(w.shape)}")
        sino = sino.contiguous()
        filt = torch.empty_like(sino)
        N.check(N.lib.rn_filter_weighted(_dev_ptr(filt), _dev_ptr(sino), _dev_ptr(w), B, C, nu, nview, nv,
                                          float(geom.da), float(geom.off_a), float(geom.dsd), float(geom.dso),
                                          int(type_filter), 1, _stream_ptr(sino.device)))
    return plan.backproject(filt, N.RN_TYPE_PIXEL, out=out)


def tv_iso_sqs(img: torch.Tensor, ndim: int, eps: float = 1e-8, want_var: bool = True):
    """Isotropic TV surrogate (PriorFunctionSolver/TVSQS.cu) of a CUDA tensor
    [nb, nx, ny, nc] (ndim 2) or [nb, nx, ny, nz, nc] (ndim 3) -> (s1, s2, var)."""
    if ndim == 2:
        nb, nx, ny, nc = img.shape
        nz = 1
    else:
        nb, nx, ny, nz, nc = img.shape
    img = img.contiguous()
    s1, s2 = torch.empty_like(img), torch.empty_like(img)
    var = torch.empty_like(img) if want_var else None
    N.check(N.lib.rn_tv_iso_sqs(_dev_ptr(s1), _dev_ptr(s2), _dev_ptr(var) if var is not None else None,
                                _dev_ptr(img), nb, nx, ny, nz, nc, float(eps), int(ndim), _stream_ptr(img.device)))
    return s1, s2, var


def tv_sqs(img: torch.Tensor, want_tv: bool = True):
    """TV surrogate terms of a [S, nx, ny] CUDA tensor -> (grad, norm, tv[S] float64)."""
    S, nx, ny = img.shape
    grad = torch.empty_like(img)
    norm = torch.empty_like(img)
    tv = torch.empty(S, dtype=torch.float64, device=img.device) if want_tv else None
    N.check(N.lib.rn_tv_sqs(_dev_ptr(grad), _dev_ptr(norm), tv.data_ptr() if tv is not None else None,
                            _dev_ptr(img), S, nx, ny, _stream_ptr(img.device)))
    return grad, norm, tv


class CylPlan:
    """Native plan of the cylindrical-detector cone-beam DD pair (rn_cyl_*):
    volumes [B, nx, ny, nz], projections [B, nu, nview, nv], float32 CUDA
    tensors; kernels run on the current stream of the plan's device."""

    def __init__(self, geom: CylGeometry, angles, nbatches: int = 1, device=None):
        self.geom = geom
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.angles = np.ascontiguousarray(np.asarray(angles, np.float32).ravel())
        self.nbatches = int(nbatches)
        self._plan = ctypes.c_void_p()
        g = geom.native(self.nbatches, self.angles.size)
        with torch.cuda.device(self.device):
            N.check(N.lib.rn_cyl_plan_create(ctypes.byref(self._plan), ctypes.byref(g),
                                             self.angles.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                             _stream_ptr(self.device)))
        self.vol_shape = (self.nbatches, geom.nx, geom.ny, geom.nz)
        self.prj_shape = (self.nbatches, geom.nu, self.angles.size, geom.nv)

    def __del__(self):
        if getattr(self, "_plan", None) and self._plan.value:
            N.lib.rn_cyl_plan_destroy(self._plan)
            self._plan = ctypes.c_void_p()

    def _check(self, t, shape):
        if tuple(t.shape) != shape or t.dtype != torch.float32 or not t.is_contiguous() or t.device != self.device:
            raise ValueError(f"expected a contiguous float32 tensor of shape {shape} on {self.device}")

    def project(self, vol: torch.Tensor, out: Optional[torch.Tensor] = None) -> torch.Tensor:
        self._check(vol, self.vol_shape)
        out = torch.empty(self.prj_shape, device=self.device) if out is None else out
        self._check(out, self.prj_shape)
        N.check(N.lib.rn_cyl_project(self._plan, _dev_ptr(out), _dev_ptr(vol), _stream_ptr(self.device)))
        return out

    def backproject(self, prj: torch.Tensor, out: Optional[torch.Tensor] = None) -> torch.Tensor:
        self._check(prj, self.prj_shape)
        out = torch.empty(self.vol_shape, device=self.device) if out is None else out
        self._check(out, self.vol_shape)
        N.check(N.lib.rn_cyl_backproject(self._plan, _dev_ptr(out), _dev_ptr(prj), _stream_ptr(self.device)))
        return out

    def launches(self) -> int:
        return int(N.lib.rn_cyl_plan_launches(self._plan))
