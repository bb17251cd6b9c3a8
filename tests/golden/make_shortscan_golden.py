"""Golden vectors for the short-scan weights from the reference's own Python.

The reference's ParkerWeighting / RiessWeighting are plain numpy + scipy
functions (python/ReconNet_no_tf.py:640-693), but importing that module loads
its CUDA library at import time.  This script therefore reads the source file,
takes only those two function definitions from its syntax tree, runs them with
numpy (see _NumpyOfItsTime) and scipy on a few short-scan geometries, and writes
tests/golden/ref_shortscan.npz.  It runs where a checkout of the reference is
present (set RECONNET_REFERENCE to it); nothing at test time reads the
reference.

    RECONNET_REFERENCE=<checkout> python tests/golden/make_shortscan_golden.py
"""
import ast
import os
import sys
from types import SimpleNamespace

import numpy as np
import scipy.ndimage

HERE = os.path.dirname(os.path.abspath(__file__))


class _NumpyOfItsTime:
    """numpy as the reference was written against.  RiessWeighting calls
    np.where on the 0-d result of np.all (python/ReconNet_no_tf.py:687).
    numpy up to 1.x treated a 0-d condition as a 1-element array (index [0]
    when true, none when false) with a deprecation warning; numpy 2 raises.
    This proxy restores the old reading for that one case and forwards
    everything else to numpy unchanged."""

    def __getattr__(self, name):
        return getattr(np, name)

    @staticmethod
    def where(cond, *args):
        if not args and np.ndim(cond) == 0:
            return np.atleast_1d(cond).nonzero()
        return np.where(cond, *args)


def load_reference_functions(root):
    path = os.path.join(root, "python", "ReconNet_no_tf.py")
    tree = ast.parse(open(path).read(), filename=path)
    keep = [n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name in ("ParkerWeighting", "RiessWeighting")]
    assert len(keep) == 2, "reference functions not found"
    ns = {"np": _NumpyOfItsTime(), "scipy": scipy}
    exec(compile(ast.Module(body=keep, type_ignores=[]), path, "exec"), ns)
    return ns["ParkerWeighting"], ns["RiessWeighting"]


CASES = [
    # name, nu, da, off_a, nview, extra over-scan (rad) beyond the fan
    ("c736", 736, 1.2858 / 1085.6, 0.0, 150, 0.0),
    ("c736_off", 736, 1.2858 / 1085.6, 1.25, 97, 0.05),
    ("c96", 96, 0.0022, -0.25, 120, 0.0),
    ("c200_wide", 200, 0.004, 0.0, 121, 0.2),
]


def main():
    root = os.environ.get("RECONNET_REFERENCE")
    if not root:
        sys.exit("set RECONNET_REFERENCE to a checkout of the reference")
    parker, riess = load_reference_functions(root)
    out = {}
    for name, nu, da, off_a, nview, extra in CASES:
        fan = nu * da
        ang = (np.arange(nview) * (np.pi + fan + extra) / (nview - 1)).astype(np.float32)
        # float32 angle values held in float64: under numpy 2's promotion rules
        # float32 scalars would pull the weight arithmetic down to float32,
        # which the float64 arithmetic of the numpy the reference was written
        # for did not do
        rn = SimpleNamespace(nu=nu, da=da, off_a=off_a, angles=ang.astype(np.float64))
        out[f"{name}_angles"] = ang
        out[f"{name}_geom"] = np.array([nu, da, off_a], np.float64)
        out[f"{name}_parker"] = np.asarray(parker(rn), np.float32)[0, :, :, 0]
        out[f"{name}_riess"] = np.asarray(riess(rn), np.float32)[0, :, :, 0]
        out[f"{name}_riess_s12"] = np.asarray(riess(rn, sigma=12, theta=0.1), np.float32)[0, :, :, 0]
    np.savez_compressed(os.path.join(HERE, "ref_shortscan.npz"), **out)
    print("wrote", os.path.join(HERE, "ref_shortscan.npz"), len(out), "arrays")


if __name__ == "__main__":
    main()
