"""Golden vectors for the oracle's model of the texture unit (GPU machine).

Builds, from the fan2d golden case, the reference's two prefix-sum textures
(FP32 serial prefix sums along x and y, as AccumulateKernelX/Y do,
ReconNet4D/DistanceDriven.cu:23-60) and the fetch coordinates of its X- and
Y-class forward kernels (row / column integer, prefix fractional), plus a
sweep of impulse fetches over pairs of fractional coordinates; fetches them
through tests/golden/texfetch.cu on the GPU and writes
tests/golden/ref_texfetch.npz.

    nvcc -gencode arch=compute_100a,code=sm_100a -o /tmp/texfetch tests/golden/texfetch.cu
    python tests/golden/make_texfetch_golden.py /tmp/texfetch [outdir]
"""
import os
import struct
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def run(exe, table, modes, coords):
    D, H, W = table.shape
    with tempfile.TemporaryDirectory() as td:
        fi, fo = os.path.join(td, "in.bin"), os.path.join(td, "out.bin")
        with open(fi, "wb") as f:
            f.write(struct.pack("7i", W, H, D, *modes, len(coords)))
            f.write(np.ascontiguousarray(table, np.float32).tobytes())
            f.write(np.ascontiguousarray(coords, np.float32).tobytes())
        subprocess.check_call([exe, fi, fo])
        return np.fromfile(fo, np.float32)


def main():
    exe = sys.argv[1]
    outdir = sys.argv[2] if len(sys.argv) > 2 else HERE
    d = np.load(os.path.join(HERE, "ref_fan2d.npz"))
    img = d["img"][0, :, :, 0, 0].astype(np.float32)          # [nx][ny]
    nx, ny = img.shape
    px = np.zeros((nx + 1, ny), np.float32)                     # texture X: extent (1, ny, nx + 1)
    for ix in range(nx):
        px[ix + 1] = px[ix] + img[ix]
    py = np.zeros((nx, ny + 1), np.float32)                     # texture Y: extent (1, ny + 1, nx)
    for iy in range(ny):
        py[:, iy + 1] = py[:, iy] + img[:, iy]
    rng = np.random.default_rng(4)
    # X-class fetches: (0.5, row iy, x + 0.5) with x across and beyond the image
    n = 6000
    cx = np.stack([np.full(n, 0.5), rng.integers(0, ny, n).astype(np.float64),
                   rng.uniform(-3.0, nx + 4.0, n)], 1).astype(np.float32)
    vx = run(exe, px[:, :, None], (0, 0, 1), cx)
    # Y-class fetches: (0.5, y + 0.5, column ix)
    cy = np.stack([np.full(n, 0.5), rng.uniform(-3.0, ny + 4.0, n), rng.integers(0, nx, n).astype(np.float64)],
                  1).astype(np.float32)
    vy = run(exe, py[:, :, None], (0, 1, 0), cy)
    # impulse: one texel of value 1 in an 8 x 8 (h, d) texture, two fractional coordinates
    imp = np.zeros((8, 8, 1), np.float32)
    imp[4, 4, 0] = 1.0
    f = (np.arange(64) * 4 + 1.37) / 256.0
    f1, f2 = np.meshgrid(f, f, indexing="ij")
    ci = []
    for c1 in (0, 1):
        for c2 in (0, 1):
            ci.append(np.stack([np.full(f1.size, 0.5), (4 - c1) + 0.5 + f1.ravel(), (4 - c2) + 0.5 + f2.ravel()], 1))
    ci = np.concatenate(ci).astype(np.float32)
    vi = run(exe, imp, (0, 0, 1), ci)
    np.savez_compressed(os.path.join(outdir, "ref_texfetch.npz"), px=px, py=py, cx=cx, vx=vx, cy=cy, vy=vy, ci=ci, vi=vi)
    print("wrote ref_texfetch.npz")


if __name__ == "__main__":
    main()
