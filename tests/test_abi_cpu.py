"""CPU checks of the C ABI: the shared library loads, exports every symbol that
include/reconnet_b200.h declares, and rejects bad arguments before touching a
GPU (no compute calls here)."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "reconnet_b200.h")


def _declared():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?(?:int|void|float|char|int64_t|long long)\s*\**\s*(\w+)\s*\(", src, re.M)))


def test_library_builds_and_loads():
    from reconnet_b200 import _native as N
    assert os.path.exists(N.LIB_PATH)
    assert N.lib.rn_version() >= 1


def test_every_declared_symbol_is_exported():
    from reconnet_b200 import _native as N
    names = _declared()
    assert len(names) >= 25
    out = subprocess.run(["nm", "-D", "--defined-only", N.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(l.split()[-1] for l in out.splitlines() if " T " in l)
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    assert set(names) == set(N.SIGNATURES)   # the Python binding covers the whole header


def test_reference_signatures_match_reference_python_calls():
    """The drop-in names take the argument counts the reference's ctypes
    wrapper passes (python/ReconNet_no_tf.py:133-288, 396-440, 612-628)."""
    from reconnet_b200 import _native as N
    counts = {"cDistanceDrivenFanProjection": 21, "cDistanceDrivenFanBackprojection": 21,
              "cDistanceDrivenTomoProjection": 22, "cDistanceDrivenTomoBackprojection": 22,
              "cFilterFanFilter": 15, "cFilterParallelFilter": 15, "cOSSQS": 29, "cTVSQS2D": 5, "SetDevice": 1,
              "cSiddonFanProjection": 21, "cSiddonFanBackprojection": 21, "cPixelDrivenFanBackprojection": 21,
              "cSiddonConeProjectionAbitrary": 24, "cSiddonConeBackprojectionAbitrary": 24,
              "cOSSQSConeAbitrary": 33}
    for k, n in counts.items():
        assert len(N.SIGNATURES[k][1]) == n, k


def test_bad_geometry_rejected_without_gpu():
    from reconnet_b200 import _native as N
    g = N.RnFanGeom()
    g.nBatches = g.nChannels = 1
    g.nx = g.ny = 0          # invalid
    g.nz = g.nu = g.nview = g.nv = 1
    plan = ctypes.c_void_p()
    ang = np.zeros(1, np.float32)
    st = N.lib.rn_fan_plan_create(ctypes.byref(plan), ctypes.byref(g),
                                  ang.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), None)
    assert st == N.RN_ERR_ARG
    assert "positive" in N.last_error()
    assert N.lib.rn_fan_project(None, None, None, None) == N.RN_ERR_ARG
    assert N.lib.rn_fan_backproject(None, None, None, 2, 0, None) == N.RN_ERR_ARG
    assert N.lib.rn_fan_sqs_update(None, None, None, None, None, None, 1.0, 0.0, 1, 0.0, 1.0, 9, None) == N.RN_ERR_ARG


def test_tuning_calls_reject_null_plans_without_gpu():
    from reconnet_b200 import _native as N
    v = ctypes.c_int()
    assert N.lib.rn_fan_plan_autotune(None, None, None, 2, None) == N.RN_ERR_ARG
    assert N.lib.rn_fan_plan_set_tuning(None, 0, 0, 0, None) == N.RN_ERR_ARG
    assert N.lib.rn_fan_plan_get_tuning(None, ctypes.byref(v), ctypes.byref(v), ctypes.byref(v)) == N.RN_ERR_ARG
    assert "null" in N.last_error()


def test_reference_named_void_calls_report_errors():
    from reconnet_b200 import _native as N
    fp = ctypes.POINTER(ctypes.c_float)()
    N.lib.cDistanceDrivenFanProjection(fp, fp, fp, 1, 1, 4, 4, 1, 1, 1, 1, 8, 4, 1, 0.01, 1, 0, 0, 1085.6, 595.0, 0)
    assert N.lib.rn_last_status() == N.RN_ERR_ARG
    with pytest.raises(N.ReconNetError):
        N.check_last()


def test_prior_shim_exports_reference_names():
    """libreconnet_b200_prior.so exports the prior solver's cTVSQS2D /
    cTVSQS3D (include/reconnet_b200_prior.h) and resolves its forwarder."""
    import re
    from conftest import ROOT
    from reconnet_b200 import _native as N
    hdr = open(os.path.join(ROOT, "include", "reconnet_b200_prior.h")).read()
    names = set(re.findall(r"^void (\w+)\(", hdr, re.M))
    assert names == set(N.PRIOR_SIGNATURES)
    lib = N.prior_lib()
    for n in names:
        assert hasattr(lib, n)
