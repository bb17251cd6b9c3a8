import os
import sys
from types import SimpleNamespace

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); parity tests through the C ABI")


def pytest_collection_modifyitems(config, items):
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def small_fan(**kw):
    """A small fan geometry that still exercises both view classes, the fan
    edges and the image border: 48x40 image (non-square), 64 channels."""
    base = dict(nx=48, ny=40, nz=1, dx=1.0, dy=1.1, dz=1.0, nu=64, nv=1, da=0.0025, dv=1.0,
                off_a=0.0, off_v=0.0, dsd=1085.6, dso=595.0, cx=0.0, cy=0.0, cz=0.0)
    base.update(kw)
    return SimpleNamespace(**base)


def to_geometry(ns):
    from reconnet_b200.torch_ops import FanGeometry
    return FanGeometry(**{k: getattr(ns, k) for k in FanGeometry.__dataclass_fields__})


@pytest.fixture
def rng():
    return np.random.default_rng(1234)
