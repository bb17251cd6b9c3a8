"""Host-side logic that needs no GPU: the reference-mirroring ReconNet class,
subset construction, the torch TV terms, seeded inputs, and the
multi-process slice sharding of the benchmark (gloo, world size 2)."""
import os
import socket

import numpy as np
import pytest

from conftest import rel_l2


def test_reconnet_defaults_and_from_file(tmp_path):
    from reconnet_b200.reconnet import ReconNet
    rn = ReconNet()
    # python/ReconNet_no_tf.py:27-47
    assert (rn.nu, rn.rotview, rn.nx, rn.ny, rn.dsd, rn.dso) == (736, 720, 512, 512, 1085.6, 595)
    assert abs(rn.da - 1.2858 / 1085.6) < 1e-12
    assert len(rn.angles) == 720 and rn.angles[1] == pytest.approx(2 * np.pi / 720, rel=1e-6)
    f = tmp_path / "param.txt"
    f.write_text("nu 888\nrotview 1152\nnx 256\nDX 0.7\ndu 1.0\noff_a 0.25\n")
    rn.FromFile(str(f))
    assert rn.nu == 888 and rn.rotview == 1152 and rn.nx == 256 and isinstance(rn.nu, int)
    assert rn.dx == pytest.approx(0.7)
    assert rn.off_a == pytest.approx(-0.25)           # sign flip of ReconNet_no_tf.py:68
    assert rn.da == pytest.approx(1.0 / 1085.6, rel=1e-6)
    assert len(rn.angles) == 1152


def test_shortscan_weights_oracle_shape_and_range():
    """The oracle's Parker weights lie in [0, 1] and sum, over a ray and its
    conjugate, to one; Riess weights lie in [0, 2]."""
    from oracle import oracle as O
    nu, da = 64, 0.01
    ang = np.linspace(0, np.pi + 2 * 0.4, 300).astype(np.float32)
    w = O.shortscan_weights(ang, nu, da, 0.0, "parker")
    assert w.shape == (64, 300)
    assert np.all(w >= 0) and np.all(w <= 1 + 1e-12)
    r = O.shortscan_weights(ang, nu, da, 0.0, "riess")
    assert np.all(r >= -1e-12) and np.all(r <= 2 + 1e-12)


def test_interleaved_subsets_cover_views_once():
    from reconnet_b200.ossqs import interleaved_subsets
    for nview, M in ((720, 12), (577, 24), (50, 4)):
        subs = interleaved_subsets(nview, M)
        allv = np.sort(np.concatenate(subs))
        assert np.array_equal(allv, np.arange(nview))
        assert max(len(s) for s in subs) - min(len(s) for s in subs) <= 1


def test_torch_tv_terms_match_oracle(rng):
    import torch
    from oracle import oracle as O
    from reconnet_b200.ossqs import tv_terms
    img = (rng.random((11, 9)) * 0.02).astype(np.float32)
    g, n = tv_terms(torch.from_numpy(img).double())
    g2, n2, _ = O.tv_sqs(img)
    assert rel_l2(g.numpy(), g2) < 1e-6 and rel_l2(n.numpy(), n2) < 1e-6


def test_phantom_is_seeded_and_in_range():
    from reconnet_b200 import phantom as P
    a = P.ellipse_phantom(64, 64, 1.0, 1.0, np.random.default_rng(3))
    b = P.ellipse_phantom(64, 64, 1.0, 1.0, np.random.default_rng(3))
    assert np.array_equal(a, b) and a.dtype == np.float32
    assert a.min() >= 0 and a.max() <= 0.4
    c = P.batch_view_counts(64, seed=1)
    assert c.min() >= 576 and c.max() <= 1152 and len(c) == 64
    s, w = P.poisson_sinogram(np.full((4, 5), 2.0), 1e4, np.random.default_rng(0))
    assert s.shape == (4, 5) and np.all(w >= 1)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _shard_worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    geom, counts, angles, imgs = bench.workload(rank, 4)
    import torch
    t = torch.tensor([float(counts.sum())], dtype=torch.float64)
    dist.all_reduce(t)
    ms = torch.tensor([10.0 + rank], dtype=torch.float64)
    dist.all_reduce(ms, op=dist.ReduceOp.MAX)
    q.put((rank, counts.tolist(), float(imgs.sum()), float(t.item()), float(ms.item())))
    dist.destroy_process_group()


def test_bench_shards_independent_batches_per_rank():
    """Each rank builds its own seeded batch (weak scaling, no data-path
    collective); the timing reduction is a max over ranks."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_shard_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
    assert all(p.exitcode == 0 for p in ps)
    (r0, c0, s0, tot0, ms0), (r1, c1, s1, tot1, ms1) = res
    assert c0 != c1 and s0 != s1                  # different batches per rank
    assert tot0 == tot1 == sum(c0) + sum(c1)      # all-reduce reaches every rank
    assert ms0 == ms1 == 11.0                      # max over ranks


def test_learned_schedule_choice_is_cheapest_within_target():
    """choose_schedule takes the schedule with the fewest OS-SQS iterations
    (then network passes) whose RMSE exceeds the TV reconstruction's by at
    most the allowance (0 by default: matching TV), and the lowest-RMSE one
    when none does; run_schedule applies iterations and network passes in
    the order given.  Checked with stand-ins for the solver and the network."""
    import torch
    from reconnet_b200 import learned_prior as LP

    class Net:
        def denoise(self, x):
            return x * 0.5

    class Solver:
        def run(self, x, k):
            return x + k

    x0 = torch.zeros(2, 3)
    assert float(LP.run_schedule(Net(), Solver(), x0, (4, "N", 2, "N", 2))[0, 0]) == 4.0   # ((4/2)+2)/2+2
    assert LP.schedule_cost((4, "N", 3, "N", 2)) == (9, 2)
    ref = torch.full((2, 3), 2.0)
    sch, errs, excess = LP.choose_schedule(Net(), Solver(), ref, ref + 0.25)
    assert sch == (4, "N") and errs[(4, "N")] == 0.0 and abs(excess[(4, "N")] + 0.25) < 1e-6
    # only the schedules ending in 2 iterations after two passes reach 4.0;
    # with TV 0.05 off, they alone match it
    ref4 = torch.full((2, 3), 4.0)
    sch, errs, excess = LP.choose_schedule(Net(), Solver(), ref4, ref4 + 0.05)
    assert sch == (4, "N", 2, "N", 2)
    # an allowance of 2 admits the cheapest, (4, N): 2.0 off, TV 0.05 off
    sch, errs, excess = LP.choose_schedule(Net(), Solver(), ref4, ref4 + 0.05, allowance=2.0)
    assert sch == (4, "N") and abs(excess[sch] - 1.95) < 1e-6
    # none within: the lowest RMSE
    ref100 = torch.full((2, 3), 100.0)
    sch, errs, excess = LP.choose_schedule(Net(), Solver(), ref100, ref100)
    assert errs[sch] == min(errs.values())