"""Isotropic total-variation surrogate of the reference's prior solver
(PriorFunctionSolver/TVSQS.cu), with the function names and arguments of its
Python wrapper (python/PriorFunctionSolver2.py:161-205): ``cTVSQS2D(x, eps)``
on [nb, nx, ny, nc] and ``cTVSQS3D(x, eps)`` on [nb, nx, ny, nz, nc], each
returning (s1, s2, var).  They call the prior-solver shim library
(libreconnet_b200_prior.so, the reference's C names) on host arrays; the
device form is ``reconnet_b200.torch_ops.tv_iso_sqs``."""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native as N

_fp = ctypes.POINTER(ctypes.c_float)


def _p(a):
    return a.ctypes.data_as(_fp)


def cTVSQS2D(x, eps=1e-8):
    x = np.ascontiguousarray(x, np.float32)
    if x.ndim != 4:
        raise ValueError("x must be [nb, nx, ny, nc]")
    s1, s2, var = (np.zeros(x.shape, np.float32) for _ in range(3))
    N.prior_lib().cTVSQS2D(_p(s1), _p(s2), _p(var), _p(x), *x.shape, float(eps))
    N.check_last()
    return s1, s2, var


def cTVSQS3D(x, eps=1e-8):
    x = np.ascontiguousarray(x, np.float32)
    if x.ndim != 5:
        raise ValueError("x must be [nb, nx, ny, nz, nc]")
    s1, s2, var = (np.zeros(x.shape, np.float32) for _ in range(3))
    N.prior_lib().cTVSQS3D(_p(s1), _p(s2), _p(var), _p(x), *x.shape, float(eps))
    N.check_last()
    return s1, s2, var
