"""Seeded synthetic inputs: random-ellipse phantoms, Poisson-noise sinograms and
the workload geometries (the reference's Mayo slices and param.txt are not
available; these stand in for them with the stated shapes and value ranges).
"""
from __future__ import annotations

import numpy as np

from .geometry import FanGeometry

MU_WATER = 0.019          # 1/mm
HU = MU_WATER / 1000.0    # one Hounsfield unit in 1/mm


def ellipse_phantom(nx, ny, dx, dy, rng, n_ellipses=10, axes=(5.0, 120.0), mu=(0.0, 0.04), fov_frac=0.8):
    """Sum of random ellipses on a [nx, ny] grid (index [ix, iy]); centres
    uniform within fov_frac x FOV radius, axes U[axes] mm, angles U[0, pi),
    attenuation U[mu] 1/mm, additive."""
    xs = (np.arange(nx) - (nx - 1) / 2.0) * dx
    ys = (np.arange(ny) - (ny - 1) / 2.0) * dy
    X, Y = np.meshgrid(xs, ys, indexing="ij")
    R = fov_frac * min(nx * dx, ny * dy) / 2.0
    img = np.zeros((nx, ny), np.float64)
    for _ in range(n_ellipses):
        rr = R * np.sqrt(rng.uniform())
        th = rng.uniform(0, 2 * np.pi)
        cx, cy = rr * np.cos(th), rr * np.sin(th)
        a, b = rng.uniform(*axes, size=2)
        ang = rng.uniform(0, np.pi)
        val = rng.uniform(*mu)
        c, s = np.cos(ang), np.sin(ang)
        u = (X - cx) * c + (Y - cy) * s
        v = -(X - cx) * s + (Y - cy) * c
        img[(u / a) ** 2 + (v / b) ** 2 <= 1.0] += val
    return img.astype(np.float32)


def ellipsoid_phantom(nx, ny, nz, dx, dy, dz, rng, n_ellipsoids=10, axes=(5.0, 120.0), mu=(0.0, 0.04),
                      device=None):
    """Random 3D ellipsoids on [nx, ny, nz] (axis-aligned in z, rotated in xy).
    With ``device`` (a torch device) the volume is rasterised there and
    returned as a torch tensor; the seeded parameters are the same."""
    if device is not None:
        import torch
        ar = lambda n, d: (torch.arange(n, device=device, dtype=torch.float64) - (n - 1) / 2.0) * d
        X, Y, Z = torch.meshgrid(ar(nx, dx), ar(ny, dy), ar(nz, dz), indexing="ij")
        img = torch.zeros((nx, ny, nz), dtype=torch.float32, device=device)
    else:
        xs = (np.arange(nx) - (nx - 1) / 2.0) * dx
        ys = (np.arange(ny) - (ny - 1) / 2.0) * dy
        zs = (np.arange(nz) - (nz - 1) / 2.0) * dz
        X, Y, Z = np.meshgrid(xs, ys, zs, indexing="ij")
        img = np.zeros((nx, ny, nz), np.float32)
    R = 0.8 * min(nx * dx, ny * dy) / 2.0
    for _ in range(n_ellipsoids):
        rr = R * np.sqrt(rng.uniform())
        th = rng.uniform(0, 2 * np.pi)
        cx, cy = rr * np.cos(th), rr * np.sin(th)
        cz = rng.uniform(-0.4, 0.4) * nz * dz
        a, b = rng.uniform(*axes, size=2)
        c3 = rng.uniform(axes[0], min(axes[1], nz * dz / 2))
        ang = rng.uniform(0, np.pi)
        val = rng.uniform(*mu)
        c, s = np.cos(ang), np.sin(ang)
        u = (X - cx) * c + (Y - cy) * s
        v = -(X - cx) * s + (Y - cy) * c
        img[(u / a) ** 2 + (v / b) ** 2 + ((Z - cz) / c3) ** 2 <= 1.0] += val
    return img


def poisson_sinogram(line_integrals, I0, rng):
    """b = -ln(max(Poisson(I0 exp(-Ax)), 1) / I0); weights W = counts."""
    counts = rng.poisson(I0 * np.exp(-np.asarray(line_integrals, np.float64)))
    counts = np.maximum(counts, 1).astype(np.float64)
    b = -np.log(counts / I0)
    return b.astype(np.float32), counts.astype(np.float32)


def uniform_angles(nview):
    """Angles 2*pi*k/nview as float32 (python/ReconNet_no_tf.py:73)."""
    return (np.arange(nview, dtype=np.float32) * 2 * np.pi / nview).astype(np.float32)


# ---- workload geometries ----
def geom_fan256() -> FanGeometry:
    """256x256 1.0 mm image, 736-channel arc detector at 1.2858 mm, 720 views."""
    return FanGeometry(nx=256, ny=256, nz=1, dx=1.0, dy=1.0, dz=1.0, nu=736, nv=1, da=1.2858 / 1085.6, dv=1.0,
                       dsd=1085.6, dso=595.0)


def geom_fan512() -> FanGeometry:
    """512x512 0.7 mm slices, 888 channels (1.2858 mm pitch assumed)."""
    return FanGeometry(nx=512, ny=512, nz=1, dx=0.7, dy=0.7, dz=1.0, nu=888, nv=1, da=1.2858 / 1085.6, dv=1.0,
                       dsd=1085.6, dso=595.0)


def batch_view_counts(nslices=64, seed=1):
    """Seeded uneven view counts in [576, 1152] per slice."""
    rng = np.random.default_rng(seed)
    return rng.integers(576, 1153, size=nslices).astype(np.int32)
