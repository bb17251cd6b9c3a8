"""CPU checks of the oracle itself: independent restatements (pure Python /
numpy) of the reference formulas on tiny cases, the adjoint identity of the
matched pair, and FP32-port vs FP64 consistency."""
import math

import numpy as np
import pytest

from conftest import rel_l2, small_fan
from oracle import oracle as O


def _geom_tiny(**kw):
    g = small_fan(nx=12, ny=10, nu=20, da=0.004, dx=1.0, dy=1.2)
    for k, v in kw.items():
        setattr(g, k, v)
    # the C ABI takes float32 geometry: round here so the direct restatements
    # below see the same parameters
    for k in ("dx", "dy", "dz", "da", "dv", "off_a", "off_v", "dsd", "dso"):
        setattr(g, k, float(np.float32(getattr(g, k))))
    return g


def _direct_fan_fp(img2d, angles, g):
    """Pure-Python DDFPFanKernelX/Y (DistanceDriven.cu:64-196) for nz = nv = 1
    with exact interpolation: each row boundary iy blends rows iy-1 / iy
    (border row -1 = 0), the footprint integral is an explicit overlap sum."""
    nx, ny = img2d.shape
    out = np.zeros((g.nu, len(angles)))

    def row_integral(vals, x):      # integral of piecewise-constant row from 0 to clamp(x)
        x = min(max(x, 0.0), len(vals))
        k = int(math.floor(x))
        s = float(np.sum(vals[:k], dtype=np.float64))
        if k < len(vals):
            s += (x - k) * vals[k]
        return s

    for iv, th in enumerate(angles):
        xcls = O.view_is_x(th)          # float rule of DistanceDriven.cu:302
        th = float(th)
        c, s = math.cos(th), math.sin(th)
        for iu in range(g.nu):
            a = (-(iu - (g.nu - 1) / 2) - g.off_a) * g.da
            src = (g.dso * s / g.dx + nx / 2, -g.dso * c / g.dy + ny / 2)
            ends = []
            for da in (-g.da / 2, g.da / 2):
                ex, ey = g.dsd * math.sin(a + da), -g.dso + g.dsd * math.cos(a + da)
                ends.append(((ex * c - ey * s) / g.dx + nx / 2, (ex * s + ey * c) / g.dy + ny / 2))
            val = 0.0
            if xcls:
                r = [(e[0] - src[0]) / (e[1] - src[1]) for e in ends]
                for iy in range(ny):
                    x1, x2 = (src[0] + rr * (iy - src[1]) for rr in r)
                    rows = [img2d[:, iy - 1] if iy > 0 else np.zeros(nx), img2d[:, iy]]
                    d = sum(0.5 * (row_integral(rw, x2) - row_integral(rw, x1)) for rw in rows)
                    val += d / (x2 - x1)
                val *= g.dy / abs(math.cos(th - a))
            else:
                r = [(e[1] - src[1]) / (e[0] - src[0]) for e in ends]
                for ix in range(nx):
                    y1, y2 = (src[1] + rr * (ix - src[0]) for rr in r)
                    cols = [img2d[ix - 1, :] if ix > 0 else np.zeros(ny), img2d[ix, :]]
                    d = sum(0.5 * (row_integral(cl, y2) - row_integral(cl, y1)) for cl in cols)
                    val += d / (y2 - y1)
                val *= g.dx / abs(math.sin(th - a))
            out[iu, iv] = val
    return out


def test_fp_matches_direct_restatement(rng):
    g = _geom_tiny(off_a=0.3)
    img = rng.random((g.nx, g.ny)).astype(np.float32)
    ang = np.array([0.1, 0.7853982, 1.3, 2.2, 3.3, 4.0, 5.5], np.float32)
    ref = _direct_fan_fp(img.astype(np.float64), ang, g)
    got = O.fan_fp(img[None, :, :, None, None], ang, g, g.nu, 1)[0, :, :, 0, 0]
    assert rel_l2(got, ref) < 1e-12


def _direct_bp_ref(sino, angles, g, fbp):
    """Pure-Python DDBPFanKernelX/Y (DistanceDriven.cu:441-614), nz = nv = 1."""
    nu, nview = sino.shape
    out = np.zeros((g.nx, g.ny))
    for iv, th in enumerate(angles):
        xcls = O.view_is_x(th)
        th = float(th)
        c, s = math.cos(th), math.sin(th)
        w = sino[:, iv].astype(np.float64).copy()
        if not fbp:
            for iu in range(nu):
                a = (-(iu - (nu - 1) / 2) - g.off_a) * g.da
                w[iu] *= g.dy / abs(math.cos(th - a)) if xcls else g.dx / abs(math.sin(th - a))
        U = np.concatenate([[0.0], np.cumsum(w)])

        def Uat(t):   # texture fetch at t + 0.5 with clamp addressing
            k = math.floor(t)
            f = t - k
            k0, k1 = min(max(k, 0), nu), min(max(k + 1, 0), nu)
            return (1 - f) * U[k0] + f * U[k1]

        def proj(px, py):
            rx = px * c + py * s
            ry = -px * s + py * c
            return -(math.atan(rx / (ry + g.dso)) / g.da + g.off_a) + nu / 2

        for ix in range(g.nx):
            for iy in range(g.ny):
                x = (ix - (g.nx - 1) / 2) * g.dx
                y = (iy - (g.ny - 1) / 2) * g.dy
                if xcls:
                    a1, a2 = proj(x - g.dx / 2, y), proj(x + g.dx / 2, y)
                else:
                    a1, a2 = proj(x, y - g.dy / 2), proj(x, y + g.dy / 2)
                v = (Uat(a2) - Uat(a1)) / (a2 - a1)
                if fbp:
                    rx = x * c + y * s
                    ry = -x * s + y * c
                    v *= g.dso ** 2 / (rx * rx + (g.dso + ry) ** 2)
                out[ix, iy] += v
    return out


@pytest.mark.parametrize("ptype", [0, 1])
def test_bp_ref_matches_direct_restatement(rng, ptype):
    g = _geom_tiny(off_a=-0.4)
    ang = np.array([0.2, 0.7853982, 1.9, 3.0, 4.4, 5.0], np.float32)
    sino = rng.random((g.nu, ang.size)).astype(np.float32)
    ref = _direct_bp_ref(sino, ang, g, fbp=(ptype == 1))
    got = O.fan_bp(sino[None, :, :, None, None], ang, g, (g.nx, g.ny, 1), ptype)[0, :, :, 0, 0]
    assert rel_l2(got, ref) < 1e-12


@pytest.mark.parametrize("case", [
    dict(),
    dict(off_a=0.7, nx=30, ny=36),
    dict(nz=3, nv=3, dz=1.0, dv=1.0, B=2, C=2),
    dict(nz=3, nv=4, dz=1.5, dv=1.0, off_v=0.3, B=1, C=2),
])
def test_matched_bp_is_exact_transpose(rng, case):
    case = dict(case)
    B, C = case.pop("B", 1), case.pop("C", 1)
    g = small_fan(**{**dict(nx=24, ny=20, nu=40, da=0.003), **case})
    ang = np.linspace(0, 2 * np.pi, 37, endpoint=False).astype(np.float32)
    x = rng.random((B, g.nx, g.ny, g.nz, C)).astype(np.float32)
    y = rng.standard_normal((B, g.nu, ang.size, g.nv, C)).astype(np.float32)
    Ax = O.fan_fp(x, ang, g, g.nu, g.nv)
    Aty = O.fan_bp(y, ang, g, (g.nx, g.ny, g.nz), 2)
    lhs = float(np.sum(Ax * y.astype(np.float64)))
    rhs = float(np.sum(x.astype(np.float64) * Aty))
    assert abs(lhs - rhs) / abs(lhs) < 1e-12


def test_fp32_port_consistent_with_fp64(rng):
    g = small_fan()
    ang = np.linspace(0, 2 * np.pi, 30, endpoint=False).astype(np.float32)
    x = rng.random((1, g.nx, g.ny, 1, 1)).astype(np.float32)
    a64 = O.fan_fp(x, ang, g, g.nu, 1)
    a32 = O.fan_fp(x, ang, g, g.nu, 1, dtype=np.float32)
    assert rel_l2(a32, a64) < 2e-5
    y = rng.random(a64.shape).astype(np.float32)
    for t in (0, 1, 2):
        b64 = O.fan_bp(y, ang, g, (g.nx, g.ny, 1), t)
        b32 = O.fan_bp(y, ang, g, (g.nx, g.ny, 1), t, dtype=np.float32)
        assert rel_l2(b32, b64) < 2e-5


def test_fp_uniform_disk_matches_chord_lengths():
    """Physical sanity: FP of a uniform disk ~ mu * chord length (DD blurs the
    edge by about a pixel, so compare central rays only)."""
    g = small_fan(nx=128, ny=128, dx=0.5, dy=0.5, nu=96, da=0.0015)
    xs = (np.arange(g.nx) - (g.nx - 1) / 2) * g.dx
    X, Y = np.meshgrid(xs, xs, indexing="ij")
    R, mu = 25.0, 0.02
    img = (mu * (X ** 2 + Y ** 2 <= R ** 2)).astype(np.float32)
    ang = np.array([0.3, 2.0], np.float32)
    p = O.fan_fp(img[None, :, :, None, None], ang, g, g.nu, 1)[0, :, :, 0, 0]
    for iv in range(2):
        for iu in range(g.nu // 2 - 10, g.nu // 2 + 10):
            a = (-(iu - (g.nu - 1) / 2) - g.off_a) * g.da
            dist = g.dso * abs(math.sin(a))       # ray distance from the disk centre
            if dist < R - 2:
                chord = 2 * math.sqrt(R * R - dist * dist)
                assert abs(p[iu, iv] - mu * chord) < 0.02 * mu * chord


def test_ramp_kernel_matches_numpy_fft():
    nu, da = 33, float(np.float32(0.004))
    L = 2 * nu - 1
    k = np.arange(L) - (nu - 1)
    ramp = np.zeros(L)
    ramp[k == 0] = 1 / (4 * da * da)
    odd = (k % 2) != 0
    pi = 3.141592657
    ramp[odd] = -1 / (pi * pi * np.sin(k[odd] * da) ** 2)
    assert rel_l2(O.ramp_kernel(nu, da, 0), ramp) < 1e-14
    i = np.arange(L)
    wins = {1: 0.54 + 0.46 * np.cos(2 * pi * i / (L - 1)), 2: 0.5 + 0.5 * np.cos(2 * pi * i / (L - 1)),
            3: np.abs(np.cos(pi * i / (L - 1)))}
    for t, w in wins.items():
        h = np.real(np.fft.ifft(np.fft.fft(ramp) * w))
        assert rel_l2(O.ramp_kernel(nu, da, t), h) < 1e-12
    ke = -1 / (pi * pi * k[odd].astype(float) ** 2 * da * da)
    he = O.ramp_kernel(nu, da, 0, equispace=True)
    assert np.allclose(he[odd], ke)


def test_filter_matches_numpy_convolution(rng):
    g = small_fan(nu=31, da=float(np.float32(0.004)), off_a=0.25, dso=595.0)
    sino = rng.random((2, g.nu, 7, 2, 1)).astype(np.float32)
    for fan in (True, False):
        h = O.ramp_kernel(g.nu, g.da, 2, equispace=not fan)
        pw = np.cos(((np.arange(g.nu) - (g.nu - 1) / 2) - g.off_a) * g.da) if fan else np.ones(g.nu)
        scale = 3.141592657 / 7 * g.da / (g.dso if fan else 1.0)
        x = sino.astype(np.float64) * pw[None, :, None, None, None]
        ref = np.zeros_like(x)
        for iu in range(g.nu):
            ref[:, iu] = np.tensordot(h[g.nu - 1 + iu - np.arange(g.nu)], x, axes=([0], [1]))
        got = O.filter_sino(sino, g, 2, fan=fan)
        assert rel_l2(got, ref * scale) < 1e-12


def test_tv_matches_numpy(rng):
    img = rng.random((9, 7)).astype(np.float32)
    x = img.astype(np.float64)
    pad = np.pad(x, 1)
    d = [x - pad[:-2, 1:-1], x - pad[2:, 1:-1], x - pad[1:-1, :-2], x - pad[1:-1, 2:]]
    t = [np.sqrt(di * di + 1e-6) for di in d]
    grad = sum(di / ti for di, ti in zip(d, t)) / 2
    norm = sum(1 / ti for ti in t)
    tv = float(np.sum(sum(t) / 2))
    g2, n2, tv2 = O.tv_sqs(img)
    assert rel_l2(g2, grad) < 1e-6 and rel_l2(n2, norm) < 1e-6 and abs(tv2 - tv) / tv < 1e-6


def _tomo_setup(rng, nview=5):
    from types import SimpleNamespace
    g = SimpleNamespace(dx=1.0, dy=1.0, dz=2.0, cx=0.0, cy=0.0, cz=0.0, du=1.5, dv=1.5, off_u=0.2, off_v=-0.3)
    dc = np.zeros((nview, 3), np.float32)
    src = np.zeros((nview, 3), np.float32)
    for k in range(nview):
        ang = (k - (nview - 1) / 2) * 0.15
        src[k] = (600 * math.sin(ang), 10.0, 600 * math.cos(ang))
        dc[k] = (0.0, 0.0, -40.0)
    return g, dc, src


def test_tomo_pair_consistency(rng):
    """Tomo FP/BP: a constant volume projects to ~ path length * value, and BP
    of constant projections is smooth and positive."""
    g, dc, src = _tomo_setup(rng)
    nx, ny, nz, nu, nv = 16, 14, 6, 24, 20
    img = np.full((1, nx, ny, nz, 1), 0.01, np.float32)
    p = O.tomo_fp(img, dc, src, g, nu, nv)[0, :, :, :, 0]
    # central ray of the central view crosses nz*dz of material
    assert abs(p[nu // 2, 2, nv // 2] - 0.01 * nz * g.dz) < 0.01 * nz * g.dz * 0.15
    for mode in (0, 1):
        b = O.tomo_bp(np.ones((1, nu, 5, nv, 1), np.float32), dc, src, g, (nx, ny, nz), mode)
        assert np.all(b[0, 4:-4, 4:-4, :, 0] > 0)
    # weight mode 1 weights every view; mode 0 (reference) only view 0
    y = np.ones((1, nu, 5, nv, 1), np.float32)
    y[:, :, 0] = 0
    assert rel_l2(O.tomo_bp(y, dc, src, g, (nx, ny, nz), 0) * 2.0, O.tomo_bp(y, dc, src, g, (nx, ny, nz), 1)) < 0.2


def test_view_class_split_ties():
    """The class rule is evaluated in float as the reference host code does
    (DistanceDriven.cu:302): at float(3pi/4) the rounded |cos| and |sin| tie,
    so the view is Y class although |cos| > |sin| in exact arithmetic."""
    assert not O.view_is_x(np.float32(np.pi / 4))
    assert not O.view_is_x(np.float32(3 * np.pi / 4))
    d = float(np.float32(3 * np.pi / 4))
    assert abs(math.cos(d)) > abs(math.sin(d))
    assert O.view_is_x(np.float32(0.0))
    assert not O.view_is_x(np.float32(np.pi / 2))
