"""OS-SQS with a TV prior on the DD fan pair.

* ``BatchedOSSQS`` -- ordered-subset SQS for a ragged batch of independent 2D
  slices (each with its own view count): subsets interleave each slice's views
  (the reference's ``order`` mechanism, python/ReconNet_no_tf.py:419-422), one
  native plan per subset, and one full iteration (all subsets) captured in a
  CUDA graph and replayed.  The per-subset step is ``rn_fan_sqs_update``
  (ossqs.cu:91-149 arithmetic, matched backprojector, TV from
  TotalVariation.cu:9-68):

      x <- clamp(x - lam (M A_s^T W_s (A_s x - b_s) + beta grad_tv(x))
                      / (normImg + beta norm_tv(x) + 1e-6), lb, ub)

* ``unrolled_ossqs`` -- the same update unrolled for a fixed number of
  iterations with a learnable step scale and TV weight per iteration, built on
  the autograd projector pair (backward = the matched adjoint kernels) and
  checkpointed per iteration.
"""
from __future__ import annotations

from typing import Optional, Sequence

import numpy as np
import torch
import torch.utils.checkpoint as ckpt

from . import _native as N
from .torch_ops import FanGeometry, FanPlan, fan_backproject, fan_project


def interleaved_subsets(nview: int, n_subsets: int):
    """View index lists of the M interleaved subsets {m, m+M, m+2M, ...}."""
    return [np.arange(m, nview, n_subsets) for m in range(n_subsets)]


class BatchedOSSQS:
    def __init__(self, geom: FanGeometry, counts: Sequence[int], angles, sino: torch.Tensor,
                 weights: torch.Tensor, n_subsets: int, beta: float = 0.0, lam: float = 1.0,
                 lb: Optional[float] = 0.0, ub: Optional[float] = None, use_graph: bool = True,
                 device=None, projector: str = "dd", autotune: bool = True):
        """counts[s] views per slice, angles concatenated per slice, sino /
        weights packed per slice as [nu, counts[s]] blocks (flat CUDA tensors).
        projector "dd": DD forward + matched backprojection; "siddon": the
        Siddon pair, the projector of the reference's cOSSQS (ossqs.cu:81).
        autotune: time the launch parameters of the first subset's plan and
        use its choice for every subset (subsets hold ~1/n_subsets of the
        views, so their launches are much smaller than a full pass)."""
        if projector not in ("dd", "siddon"):
            raise ValueError("projector must be 'dd' or 'siddon'")
        self.type = N.RN_TYPE_SIDDON if projector == "siddon" else N.RN_TYPE_MATCHED
        self.geom = geom
        self.device = torch.device(device) if device is not None else sino.device
        self.counts = np.asarray(counts, np.int64)
        self.S = len(self.counts)
        self.M = int(n_subsets)
        if np.any(self.counts < self.M):
            raise ValueError("every slice needs at least n_subsets views")
        self.beta, self.lam = float(beta), float(lam)
        self.lb = float(np.finfo(np.float32).min) if lb is None else float(lb)
        self.ub = float(np.finfo(np.float32).max) if ub is None else float(ub)
        angles = np.asarray(angles, np.float32)
        offs = np.concatenate([[0], np.cumsum(self.counts)])
        nu = geom.nu
        # one ragged plan per subset
        self.img_shape = (self.S, geom.nx, geom.ny)
        self.plans, self.sub_b, self.sub_w = [], [], []
        for m in range(self.M):
            cnt, ang, idx = [], [], []
            for s in range(self.S):
                v = np.arange(m, self.counts[s], self.M)
                cnt.append(v.size)
                ang.append(angles[offs[s] + v])
                # element (u, k) of the subset block -> u * n_s + v_k in slice s's block
                idx.append((nu * offs[s] + np.arange(nu)[:, None] * self.counts[s] + v[None, :]).ravel())
            plan = FanPlan(geom, np.concatenate(ang), nbatches=self.S, nview_per_slice=cnt, device=self.device)
            gidx = torch.from_numpy(np.concatenate(idx)).to(self.device)
            self.plans.append(plan)
            self.sub_b.append(sino.reshape(-1)[gidx].contiguous())
            self.sub_w.append(weights.reshape(-1)[gidx].contiguous())
        if autotune:
            scratch = torch.ones(self.plans[0].img_shape, device=self.device)
            choice = self.plans[0].autotune(scratch, self.type)
            for plan in self.plans[1:]:
                plan.set_tuning(*choice)
            self.tuning = choice
        else:
            self.tuning = self.plans[0].tuning()
        # normImg = A^T W A 1 over all views (the same pair), summed over the
        # subsets in FP64: each subset's backprojection accumulates its own
        # ~1/M of the views in FP32 registers, the sum across subsets is FP64
        ones = torch.ones(self.img_shape, device=self.device)
        siddon = self.type == N.RN_TYPE_SIDDON
        norm = torch.zeros(self.img_shape, dtype=torch.float64, device=self.device)
        for m in range(self.M):
            a1 = self.plans[m].project(ones, siddon=siddon)
            norm += self.plans[m].backproject(a1 * self.sub_w[m], self.type).double()
        self.norm_img = norm.float()
        self.use_graph = use_graph
        self._graph = None
        self._xa = torch.zeros(self.img_shape, device=self.device)
        self._xb = torch.zeros(self.img_shape, device=self.device)

    def _one_iteration(self):
        src, dst = self._xa, self._xb
        for m in range(self.M):
            self.plans[m].sqs_update(dst, src, self.sub_b[m], self.sub_w[m], self.norm_img, lam=self.lam,
                                     beta=self.beta, n_subsets=self.M, lb=self.lb, ub=self.ub,
                                     type_projector=self.type)
            src, dst = dst, src
        if src is not self._xa:      # odd number of subsets: bring the result home
            self._xa.copy_(src)

    def _capture(self):
        s = torch.cuda.Stream(self.device)
        s.wait_stream(torch.cuda.current_stream(self.device))
        saved = self._xa.clone()
        with torch.cuda.stream(s):     # warm-up outside capture (lazy scratch)
            self._one_iteration()
        torch.cuda.current_stream(self.device).wait_stream(s)
        self._xa.copy_(saved)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self._one_iteration()
        self._graph = g

    def run(self, x0: torch.Tensor, n_iter: int) -> torch.Tensor:
        """n_iter full OS-SQS iterations starting from x0 ([S, nx, ny]); returns x."""
        self._xa.copy_(x0)
        if self.use_graph and self._graph is None and n_iter > 0:
            self._capture()
            self._xa.copy_(x0)
        for _ in range(n_iter):
            if self.use_graph:
                self._graph.replay()
            else:
                self._one_iteration()
        return self._xa.clone()

    def set_beta(self, beta: float) -> None:
        """Change the TV weight; the captured iteration is re-captured on the next run."""
        self.beta = float(beta)
        self._graph = None

    def check(self):
        for p in self.plans:
            p.check()


# ---------------------------------------------------------------------------
# Differentiable unrolled OS-SQS.
# ---------------------------------------------------------------------------
def tv_terms(x: torch.Tensor, eps: float = 1e-6):
    """TVSQSKernel (TotalVariation.cu:9-68) in torch on [..., nx, ny]: zero
    padding at the border, psi = sqrt(d^2 + eps); returns (grad, norm)."""
    pad = torch.nn.functional.pad(x, (1, 1, 1, 1))
    d = [x - pad[..., :-2, 1:-1], x - pad[..., 2:, 1:-1], x - pad[..., 1:-1, :-2], x - pad[..., 1:-1, 2:]]
    psi = [torch.sqrt(di * di + eps) for di in d]
    grad = sum(di / pi for di, pi in zip(d, psi)) / 2
    norm = sum(1.0 / pi for pi in psi)
    return grad, norm


def unrolled_ossqs(x0: torch.Tensor, subset_plans: Sequence[FanPlan], sub_b: Sequence[torch.Tensor],
                   sub_w: Sequence[torch.Tensor], norm_img: torch.Tensor, step_scales: torch.Tensor,
                   tv_weights: torch.Tensor, checkpoint: bool = True, bp_type: int = N.RN_TYPE_MATCHED,
                   project=None, backproject=None) -> torch.Tensor:
    """Unrolled OS-SQS in reference layout ([B, nx, ny, 1, 1] images, subset
    sinograms [B, nu, nview_s, 1, 1]); iteration k uses step scale
    step_scales[k] and TV weight tv_weights[k].  Differentiable w.r.t. x0, the
    measured data and both parameter vectors.

    bp_type is the backprojection of the update and the gradient of the
    projection: the matched transpose (exact gradients) or the reference's
    iterative backprojection (type 0, the reference's own registration,
    python/ReconNet.py:773-830).  `project(x, m)` / `backproject(r, m)`
    replace the pair (any autograd functions over subset m)."""
    M = len(subset_plans)
    if project is None:
        project = lambda x, m: fan_project(x, subset_plans[m], bp_type)
    if backproject is None:
        backproject = lambda r, m: fan_backproject(r, subset_plans[m], bp_type)

    def one_iter(x, lam, beta):
        for m in range(M):
            r = (project(x, m) - sub_b[m]) * sub_w[m]
            bp = backproject(r, m)
            g, n = tv_terms(x[..., 0, 0])
            g, n = g[..., None, None], n[..., None, None]
            x = x - lam * (M * bp + beta * g) / (norm_img + beta * n + 1e-6)
        return x

    x = x0
    for k in range(step_scales.numel()):
        if checkpoint and torch.is_grad_enabled():
            x = ckpt.checkpoint(one_iter, x, step_scales[k], tv_weights[k], use_reentrant=False)
        else:
            x = one_iter(x, step_scales[k], tv_weights[k])
    return x
