"""The view-partitioned split of one volume over ranks (reconnet_b200.
distributed), run as two gloo ranks on CPU with the FP64 oracle as each
rank's local cone-beam pair: the sharded forward projections gathered, and
the all-reduced partial backprojections, equal the single-process results."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _geom():
    from types import SimpleNamespace
    return SimpleNamespace(nx=20, ny=18, nz=6, dx=1.0, dy=1.0, dz=1.0, cx=0.0, cy=0.0, cz=0.0, nu=24, nv=5,
                           da=0.005, dv=2.0, off_a=0.0, off_v=0.0, dsd=1085.6, dso=595.0)


def _rank(rank, world, port, out):
    import sys
    sys.path.insert(0, ROOT)
    import torch
    import torch.distributed as dist
    from oracle import oracle as O
    from reconnet_b200.distributed import ViewShardedPair
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    g = _geom()
    ang = (np.arange(13) * 2 * np.pi / 13).astype(np.float32)      # 13 views: shards of 7 and 6
    rng = np.random.default_rng(0)
    vol = rng.random((1, g.nx, g.ny, g.nz)).astype(np.float32)
    y = rng.random((1, g.nu, ang.size, g.nv)).astype(np.float32)

    def make(a):
        fp = lambda v: torch.from_numpy(O.cyl_fp(v.numpy(), a, g))
        bp = lambda p: torch.from_numpy(O.cyl_bp(p.numpy().astype(np.float32), a, g, (g.nx, g.ny, g.nz)))
        return fp, bp

    pair = ViewShardedPair(ang, make)
    prj = pair.gather(pair.project(torch.from_numpy(vol)))
    back = pair.backproject(torch.from_numpy(np.ascontiguousarray(y[:, :, pair.begin:pair.end])))
    if rank == 0:
        out.put((prj.numpy(), back.numpy(), pair.shards))
    dist.barrier()
    dist.destroy_process_group()


def test_view_sharded_pair_two_gloo_ranks():
    from oracle import oracle as O
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    prj, back, shards = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert shards == [(0, 7), (7, 13)]
    g = _geom()
    ang = (np.arange(13) * 2 * np.pi / 13).astype(np.float32)
    rng = np.random.default_rng(0)
    vol = rng.random((1, g.nx, g.ny, g.nz)).astype(np.float32)
    y = rng.random((1, g.nu, ang.size, g.nv)).astype(np.float32)
    assert np.allclose(prj, O.cyl_fp(vol, ang, g), rtol=1e-12, atol=1e-12)
    assert np.allclose(back, O.cyl_bp(y, ang, g, (g.nx, g.ny, g.nz)), rtol=1e-12, atol=1e-12)


def test_view_shards_cover_every_view_once():
    from reconnet_b200.distributed import view_shards
    for nview, world in ((984, 8), (13, 2), (5, 8), (720, 3)):
        sh = view_shards(nview, world)
        assert len(sh) == world and sh[0][0] == 0 and sh[-1][1] == nview
        assert all(a[1] == b[0] for a, b in zip(sh, sh[1:]))
        sizes = [e - b for b, e in sh]
        assert max(sizes) - min(sizes) <= 1
