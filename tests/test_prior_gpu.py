"""Isotropic TV surrogate of the prior solver (PriorFunctionSolver/TVSQS.cu)
on the GPU: the device op against the FP64 oracle and the reference's own
outputs (golden vectors), and the prior-solver shim's reference-named host
entry points against the device op.  Tolerance: relative L2 <= 1e-6."""
import glob
import os

import numpy as np
import pytest

from conftest import ROOT, rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-6


@pytest.mark.parametrize("ndim,shape", [(2, (3, 37, 29, 1)), (2, (1, 1, 5, 2)), (3, (2, 13, 11, 9, 2)),
                                        (3, (1, 4, 1, 6, 1))])
def test_tv_iso_matches_oracle(ndim, shape, rng):
    import torch
    from oracle import oracle as O
    from reconnet_b200.torch_ops import tv_iso_sqs
    x = rng.random(shape).astype(np.float32)
    x[..., :2, :] = 0.25          # flat region: differences of zero
    s1, s2, var = tv_iso_sqs(torch.from_numpy(x).cuda(), ndim)
    r1, r2, rv = O.tv_iso_sqs(x, ndim)
    assert rel_l2(var.cpu().numpy(), rv) <= TOL
    assert rel_l2(s2.cpu().numpy(), r2) <= TOL
    assert rel_l2(s1.cpu().numpy(), r1) <= TOL


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(ROOT, "tests", "golden", "ref_tviso*.npz"))))
def test_tv_iso_shim_matches_reference(path):
    from reconnet_b200.prior import cTVSQS2D, cTVSQS3D
    d = dict(np.load(path))
    fn = cTVSQS2D if int(d["ndim"]) == 2 else cTVSQS3D
    s1, s2, var = fn(d["img"], float(d["eps"]))
    assert rel_l2(var, d["var"]) <= TOL
    assert rel_l2(s2, d["s2"]) <= TOL
    assert rel_l2(s1, d["s1"]) <= TOL


def test_tv_iso_shim_matches_device(rng):
    import torch
    from reconnet_b200.prior import cTVSQS3D
    from reconnet_b200.torch_ops import tv_iso_sqs
    x = rng.random((2, 9, 8, 7, 1)).astype(np.float32)
    got = cTVSQS3D(x)
    dev = tv_iso_sqs(torch.from_numpy(x).cuda(), 3)
    for a, b in zip(got, dev):
        np.testing.assert_array_equal(a, b.cpu().numpy())


def test_tv_iso_bad_arguments():
    import torch
    from reconnet_b200 import _native as N
    from reconnet_b200.torch_ops import tv_iso_sqs
    with pytest.raises(N.ReconNetError):
        tv_iso_sqs(torch.zeros((1, 4, 4, 2, 1), device="cuda"), 4)
