"""The learned prior: a 5-layer residual CNN of 3x3 convolutions (32
channels, ReLU; one channel in, one out plus the input) run, trained and
differentiated by the project's own tcgen05 tensor-core kernels
(csrc/conv.cu: forward, input gradient and weight gradient with FP32
accumulation, BF16 weights and activations).

It stands in for the TV proximal step of OS-SQS: a few OS-SQS iterations
followed by the network (``learned_ossqs``) against plain TV-SQS, which stays
the fallback and the yardstick of the image RMSE.  The reference has no CNN; its
learned use of the projectors runs through TensorFlow with the projector pair
as differentiable ops (python/ReconNet.py:773-830).

Layouts: images fp32 [N, H, W]; activations bf16 "blocked" [N, C/8, H, W, 8]
(16-byte runs of 8 channels per pixel), the layout the kernels' TMA tiles read.
The network works on normalised images u = img * ``scale`` (attenuation in
units of 1/scale mm^-1).
"""
from __future__ import annotations

import math
from typing import List, Optional, Sequence

import numpy as np
import torch

from . import _native as N

CH = 32
LAYERS = 5


def _ptr(t: Optional[torch.Tensor]) -> Optional[int]:
    return None if t is None else t.data_ptr()


def _stream(dev) -> int:
    return torch.cuda.current_stream(dev).cuda_stream


def pack_weights(w: torch.Tensor) -> torch.Tensor:
    """Forward-convolution operand image of weights w [cout, 3, 3, cin]
    (cin 1..8 -> padded to 8, or 32; cout 1 -> padded to 16, or 32): chunk kc
    x output row x 8 input channels, bf16; kc = tap * 4 + ci / 8 (cin 32) or
    kc = tap with a zero tenth chunk (cin <= 8)."""
    cout, _, _, cin = w.shape
    npad = 32 if cout == 32 else 16
    taps = w.reshape(cout, 9, cin).float()
    if cin == 32:
        img = taps.reshape(cout, 9, 4, 8).permute(1, 2, 0, 3).reshape(36, cout, 8)
    else:
        t8 = torch.zeros(cout, 9, 8, device=w.device)
        t8[:, :, :cin] = taps
        img = torch.cat([t8.permute(1, 0, 2), torch.zeros(1, cout, 8, device=w.device)], 0)
    out = torch.zeros(img.shape[0], npad, 8, device=w.device)
    out[:, :cout] = img
    return out.to(torch.bfloat16).contiguous()


def pack_dgrad_weights(w: torch.Tensor) -> torch.Tensor:
    """Operand image of the input-gradient convolution of a layer with
    weights w [cout, 3, 3, cin]: the taps reversed and the channel roles
    exchanged, so dX = conv(dY, w')."""
    return pack_weights(w.flip(1, 2).permute(3, 1, 2, 0).contiguous())


def to_blocked(x: torch.Tensor) -> torch.Tensor:
    """[N, C, H, W] (C a multiple of 8) -> bf16 blocked [N, C/8, H, W, 8]."""
    n, c, h, w = x.shape
    return x.reshape(n, c // 8, 8, h, w).permute(0, 1, 3, 4, 2).contiguous().to(torch.bfloat16)


def from_blocked(x: torch.Tensor) -> torch.Tensor:
    n, c8, h, w, _ = x.shape
    return x.permute(0, 1, 4, 2, 3).reshape(n, c8 * 8, h, w).float()


class ConvKernels:
    """Thin device calls of csrc/conv.cu on the current stream (one error word per device)."""

    def __init__(self, device):
        self.device = torch.device(device)
        self.err = torch.zeros(1, dtype=torch.int32, device=self.device)
        self.partial = None

    def conv(self, x: torch.Tensor, wpack: torch.Tensor, bias: Optional[torch.Tensor], cin: int, cout: int,
             mode: int, aux: Optional[torch.Tensor] = None, out: Optional[torch.Tensor] = None) -> torch.Tensor:
        n, _, h, w, _ = x.shape
        if out is None:
            if mode in (0, 2):
                out = torch.empty((n, cout // 8, h, w, 8), dtype=torch.bfloat16, device=self.device)
            elif mode == 1:
                out = torch.empty((n, h, w), device=self.device)
            else:
                out = torch.empty((n, cout, h, w), device=self.device)
        N.check(N.lib.rn_conv3x3(_ptr(out), _ptr(x), _ptr(wpack), _ptr(bias), _ptr(aux), n, h, w, cin, cout, mode,
                                 _ptr(self.err), _stream(self.device)))
        return out

    def wgrad(self, x: torch.Tensor, dy: torch.Tensor, cin: int, cout: int) -> torch.Tensor:
        """[32, ncols] fp32 (see rn_conv3x3_wgrad)."""
        n, _, h, w, _ = x.shape
        ncols = int(N.lib.rn_conv3x3_wgrad_cols(cin))
        nsm = torch.cuda.get_device_properties(self.device).multi_processor_count
        need = nsm * 32 * ncols
        if self.partial is None or self.partial.numel() < need:
            self.partial = torch.empty(need, device=self.device)
        out = torch.empty((32, ncols), device=self.device)
        N.check(N.lib.rn_conv3x3_wgrad(_ptr(out), _ptr(self.partial), self.partial.numel() * 4, _ptr(x), _ptr(dy), n, h,
                                       w, cin, cout, _ptr(self.err), _stream(self.device)))
        return out

    def pack_image(self, img: torch.Tensor, scale: float = 1.0, sub: Optional[torch.Tensor] = None) -> torch.Tensor:
        n, h, w = img.shape
        out = torch.empty((n, 1, h, w, 8), dtype=torch.bfloat16, device=self.device)
        N.check(N.lib.rn_conv_pack_image(_ptr(out), _ptr(img), _ptr(sub), float(scale), n, h, w, _stream(self.device)))
        return out

    def check(self):
        e = int(self.err.item())
        if e:
            self.err.zero_()
            raise N.ReconNetError(e, "a tensor-core convolution's device wait ran out")


def unpack_wgrad(g: torch.Tensor, cin: int, cout: int):
    """rn_conv3x3_wgrad columns -> (dW [cout, 3, 3, cin], db [cout])."""
    if cin == 32:
        dw = g[:cout, :288].reshape(cout, 9, 32)
        db = g[:cout, 288]
    else:
        t = torch.arange(9, device=g.device)[:, None]
        cols = (t // 2) * 16 + (t % 2) * 8 + torch.arange(8, device=g.device)[None, :]
        dw = g[:cout, cols.reshape(-1)].reshape(cout, 9, 8)
        db = g[:cout, 80]
    return dw.reshape(cout, 3, 3, -1).contiguous(), db.contiguous()


class PriorCNN:
    """The residual CNN: u -> u + f(u), f = conv5(relu(conv4(...relu(conv1(u))))).
    FP32 master weights; BF16 operand images repacked after each update."""

    def __init__(self, device="cuda", seed: int = 0, scale: float = 50.0):
        self.device = torch.device(device)
        self.scale = float(scale)
        g = torch.Generator(device="cpu").manual_seed(seed)
        self.shapes = [(CH, 1), (CH, CH), (CH, CH), (CH, CH), (1, CH)]
        self.w: List[torch.Tensor] = []
        self.b: List[torch.Tensor] = []
        for li, (co, ci) in enumerate(self.shapes):
            std = math.sqrt(2.0 / (9 * ci)) * (0.1 if li == LAYERS - 1 else 1.0)
            self.w.append((torch.randn(co, 3, 3, ci, generator=g) * std).to(self.device))
            self.b.append(torch.zeros(co, device=self.device))
        self.k = ConvKernels(self.device)
        self.adam_m = [torch.zeros_like(t) for t in self.w + self.b]
        self.adam_v = [torch.zeros_like(t) for t in self.w + self.b]
        self.adam_t = 0
        self.repack()

    def repack(self):
        self.pk = [pack_weights(w) for w in self.w]
        self.pkd = [pack_dgrad_weights(w) for w in self.w]

    def state_dict(self):
        return {f"w{i}": w.cpu().numpy() for i, w in enumerate(self.w)} | \
               {f"b{i}": b.cpu().numpy() for i, b in enumerate(self.b)} | {"scale": np.float64(self.scale)}

    def load_state_dict(self, d):
        for i in range(LAYERS):
            self.w[i] = torch.as_tensor(np.asarray(d[f"w{i}"]), dtype=torch.float32, device=self.device).contiguous()
            self.b[i] = torch.as_tensor(np.asarray(d[f"b{i}"]), dtype=torch.float32, device=self.device).contiguous()
        self.scale = float(d["scale"])
        self.repack()

    # u: normalised images [N, H, W] fp32
    def forward(self, u: torch.Tensor, keep: bool = False):
        x0 = self.k.pack_image(u)
        acts = [x0]
        a = self.k.conv(x0, self.pk[0], self.b[0], 8, CH, 0)
        acts.append(a)
        for li in (1, 2, 3):
            a = self.k.conv(a, self.pk[li], self.b[li], CH, CH, 0)
            acts.append(a)
        out = self.k.conv(a, self.pk[4], self.b[4], CH, 1, 1, aux=u)
        return (out, acts) if keep else out

    def backward(self, acts, d_out: torch.Tensor):
        """Gradients (dW list, db list) of sum(d_out * out) with respect to the weights."""
        dy = self.k.pack_image(d_out)
        dws, dbs = [None] * LAYERS, [None] * LAYERS
        g = self.k.wgrad(acts[4], dy, CH, 8)
        dws[4], dbs[4] = unpack_wgrad(g, CH, 1)
        d = self.k.conv(dy, self.pkd[4], None, 8, CH, 2, aux=acts[4])
        for li in (3, 2, 1):
            g = self.k.wgrad(acts[li], d, CH, CH)
            dws[li], dbs[li] = unpack_wgrad(g, CH, CH)
            d = self.k.conv(d, self.pkd[li], None, CH, CH, 2, aux=acts[li])
        g = self.k.wgrad(acts[0], d, 8, CH)
        dws[0], dbs[0] = unpack_wgrad(g, 8, CH)
        dws[0] = dws[0][..., :1].contiguous()     # the image is channel 0 of the 8-channel input
        return dws, dbs

    def adam_step(self, dws, dbs, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
        self.adam_t += 1
        params = self.w + self.b
        grads = list(dws) + list(dbs)
        c1 = 1 - b1 ** self.adam_t
        c2 = 1 - b2 ** self.adam_t
        for p, gr, m, v in zip(params, grads, self.adam_m, self.adam_v):
            m.mul_(b1).add_(gr, alpha=1 - b1)
            v.mul_(b2).addcmul_(gr, gr, value=1 - b2)
            p.addcdiv_(m / c1, (v / c2).sqrt_().add_(eps), value=-lr)
        self.repack()

    def denoise(self, img: torch.Tensor) -> torch.Tensor:
        """img [N, H, W] fp32 (1/mm) -> the network's output in the same units."""
        return self.forward(img.contiguous() * self.scale) / self.scale

    def train(self, inputs: torch.Tensor, targets: torch.Tensor, steps: int, batch: int = 8, lr: float = 1e-3,
              seed: int = 0, log_every: int = 0, lr_final: float = 0.01, augment: bool = True) -> List[float]:
        """Adam on the mean squared error of u_in -> u_target (normalised).
        The learning rate decays from lr to lr * lr_final on a cosine; with
        augment, each batch is taken in one of the square's eight orientations
        (a full-circle scan with uniform views treats them alike)."""
        g = torch.Generator(device="cpu").manual_seed(seed)
        n = inputs.shape[0]
        square = inputs.shape[1] == inputs.shape[2]
        losses = []
        for s in range(steps):
            idx = torch.randint(0, n, (batch,), generator=g).to(self.device)
            u = inputs[idx] * self.scale
            t = targets[idx] * self.scale
            if augment:
                o = int(torch.randint(0, 8 if square else 4, (1,), generator=g))
                if o & 1:
                    u, t = u.flip(1), t.flip(1)
                if o & 2:
                    u, t = u.flip(2), t.flip(2)
                if o & 4:
                    u, t = u.transpose(1, 2), t.transpose(1, 2)
            u, t = u.contiguous(), t.contiguous()
            out, acts = self.forward(u, keep=True)
            diff = out - t
            loss = float((diff * diff).mean()) if (log_every and s % log_every == 0) or s == steps - 1 else None
            d_out = (2.0 / diff.numel()) * diff
            dws, dbs = self.backward(acts, d_out.contiguous())
            frac = s / max(steps - 1, 1)
            self.adam_step(dws, dbs, lr=lr * (lr_final + (1 - lr_final) * 0.5 * (1 + math.cos(math.pi * frac))))
            if loss is not None:
                losses.append(loss)
        self.k.check()
        return losses


# ---------------------------------------------------------------------------
# Data and the learned-prior reconstruction
# ---------------------------------------------------------------------------
def simulate(geom, nview: int, truth: torch.Tensor, I0: float, seed: int):
    """Projections of a batch of slices [S, nx, ny] over nview uniform views
    with Poisson counts at I0: (solver angles, b, w) in the ragged packed
    layout of BatchedOSSQS (flat [S * nu * nview])."""
    from .phantom import uniform_angles
    from .torch_ops import FanPlan
    S = truth.shape[0]
    ang = np.tile(uniform_angles(nview), S)
    plan = FanPlan(geom, ang, nbatches=S, nview_per_slice=[nview] * S, device=truth.device)
    gen = torch.Generator(device=truth.device).manual_seed(seed)
    with torch.no_grad():
        line = plan.project(truth.contiguous())
        counts = torch.poisson(I0 * torch.exp(-line.double()), generator=gen).clamp_min(1.0)
        b = (-torch.log(counts / I0)).float()
    return ang, b, counts.float()


def tv_weight(solver) -> float:
    """TV weight of the OS-SQS runs: 5% of the median data curvature against
    the TV curvature of a flat image (the weight the benchmark's OS-SQS uses)."""
    from .ossqs import tv_terms
    _, n_flat = tv_terms(torch.zeros((1, 8, 8), device=solver.norm_img.device))
    return float(0.05 * solver.norm_img.median() / n_flat[0, 4, 4])


def os_sqs(geom, nview, ang, b, w, S, n_iter, n_subsets=24, beta=None, x0=None):
    """TV OS-SQS (BatchedOSSQS, graph-replayed iterations) on S slices."""
    from .ossqs import BatchedOSSQS
    solver = BatchedOSSQS(geom, [nview] * S, ang, b, w, n_subsets=n_subsets, lb=0.0, device=b.device)
    solver.beta = tv_weight(solver) if beta is None else beta
    x0 = torch.zeros((S, geom.nx, geom.ny), device=b.device) if x0 is None else x0
    x = solver.run(x0, n_iter)
    solver.check()
    return x, solver


def make_training_pairs(geom, nview: int, n_slices: int, seed: int, I0_in=1e4, I0_target=1e6, it_in=4,
                        it_target=100, n_subsets=24, chunk=32):
    """(inputs, targets, truths) [n_slices, nx, ny]: inputs = it_in OS-SQS
    iterations at I0_in, targets = it_target TV-SQS iterations at I0_target,
    on seeded random-ellipse slices."""
    from .phantom import ellipse_phantom
    rng = np.random.default_rng(seed)
    ins, tgs, tru = [], [], []
    for c0 in range(0, n_slices, chunk):
        S = min(chunk, n_slices - c0)
        truth = torch.from_numpy(np.stack([ellipse_phantom(geom.nx, geom.ny, geom.dx, geom.dy, rng)
                                           for _ in range(S)]).astype(np.float32)).cuda()
        ang, b, w = simulate(geom, nview, truth, I0_in, seed * 1000 + c0)
        x_in, _ = os_sqs(geom, nview, ang, b, w, S, it_in, n_subsets)
        ang, b, w = simulate(geom, nview, truth, I0_target, seed * 1000 + c0 + 1)
        x_tg, _ = os_sqs(geom, nview, ang, b, w, S, it_target, n_subsets)
        ins.append(x_in)
        tgs.append(x_tg)
        tru.append(truth)
    return torch.cat(ins), torch.cat(tgs), torch.cat(tru)


def learned_ossqs(net: PriorCNN, geom, nview, ang, b, w, S, n_iter=4, n_subsets=24):
    """A few OS-SQS iterations, then the network in place of the TV prior's
    remaining work; returns (image, the OS-SQS image)."""
    x, _ = os_sqs(geom, nview, ang, b, w, S, n_iter, n_subsets)
    return net.denoise(x).clamp_min_(0.0), x


# The schedules the learned path chooses from: OS-SQS iteration counts with
# "N" marking a pass of the network (its output is the next iteration's
# start).  The first entry is the path the network is trained for (its inputs
# are 4-iteration images).
SCHEDULES = ((4, "N"), (4, "N", 2, "N"), (4, "N", 2, "N", 2), (4, "N", 3, "N", 2), (4, "N", 4, "N", 2),
             (4, "N", 2, "N", 2, "N", 2))


def schedule_cost(schedule):
    """(OS-SQS iterations, network passes) of a schedule."""
    return sum(t for t in schedule if t != "N"), sum(1 for t in schedule if t == "N")


def run_schedule(net: PriorCNN, solver, x0: torch.Tensor, schedule) -> torch.Tensor:
    """Learned-prior OS-SQS: the solver's TV OS-SQS iterations (BatchedOSSQS,
    graph-replayed) interleaved with passes of the network, in the order
    `schedule` gives (see SCHEDULES)."""
    x = x0
    for t in schedule:
        x = net.denoise(x).clamp_min_(0.0) if t == "N" else solver.run(x, t)
    return x


def choose_schedule(net: PriorCNN, solver, x_ref: torch.Tensor, x_tv: torch.Tensor, allowance: float = 0.0,
                    schedules=SCHEDULES):
    """The cheapest schedule (fewest iterations, then fewest network passes)
    whose RMSE against x_ref on the solver's slices (a validation set, not the
    slices the result is reported on) exceeds that of the TV reconstruction
    x_tv by at most `allowance`; the one with the lowest RMSE if none does.
    Returns (schedule, {schedule: rmse}, {schedule: rmse - TV's rmse}).

    With the default allowance of 0 a schedule must match TV on the
    validation slices, which leaves a target of "TV + 1 HU" on other slices
    its whole tolerance as margin: a schedule's excess over TV moves from one
    set of slices to another (by ~0.6 HU between 8 validation and 32
    held-out slices here), so a schedule chosen just inside the target on
    the validation slices can miss it on the held-out ones."""
    tv = float(torch.sqrt(((x_tv - x_ref) ** 2).mean()))
    errs, excess = {}, {}
    for sch in schedules:
        x = run_schedule(net, solver, torch.zeros_like(x_ref), sch)
        errs[sch] = float(torch.sqrt(((x - x_ref) ** 2).mean()))
        excess[sch] = errs[sch] - tv
    ok = [sch for sch in schedules if excess[sch] <= allowance]
    best = min(ok, key=schedule_cost) if ok else min(schedules, key=lambda sch: errs[sch])
    return best, errs, excess