"""CPU-side checks of the C ABI library: it builds, loads without a GPU and
exports every symbol include/parflexdtw_b200.h declares (no compute calls)."""
import ctypes as ct
import os
import re

import numpy as np
import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
HEADER = os.path.join(ROOT, "include", "parflexdtw_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(pfx_\w+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    from parflexdtw_b200 import build
    path = build.build()
    return ct.CDLL(path)


def test_header_symbols_exported(lib):
    syms = declared_symbols()
    assert len(syms) >= 15
    for s in syms:
        assert hasattr(lib, s), s


def test_python_binding_covers_header():
    from parflexdtw_b200 import _lib
    bound = {name for name, _, _ in _lib.SIGNATURES}
    assert bound == set(declared_symbols())


def test_status_strings(lib):
    lib.pfx_status_string.restype = ct.c_char_p
    assert lib.pfx_status_string(4).decode().startswith("Stage 2: No valid endpoint")
    assert lib.pfx_status_string(99).decode() == "unknown status"
    lib.pfx_version.restype = ct.c_int
    assert lib.pfx_version() >= 100


def test_plan_create_without_gpu_reports_no_device(lib):
    """Without a GPU the library returns PFX_ERR_NO_DEVICE (never falls back)."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    h = ct.c_void_p()
    steps = (ct.c_int64 * 6)(1, 1, 1, 2, 2, 1)
    w = (ct.c_double * 3)(2, 3, 3)
    lib.pfx_plan_create.argtypes = [ct.c_int64, ct.c_int64, ct.c_int32,
                                    ct.POINTER(ct.c_int64), ct.POINTER(ct.c_double),
                                    ct.c_int32, ct.POINTER(ct.c_void_p)]
    assert lib.pfx_plan_create(100, 100, 20, steps, w, 3, ct.byref(h)) == 6


def test_api_refuses_cpu_path():
    import parflexdtw_b200 as pf
    C = np.abs(np.random.RandomState(0).randn(20, 20))
    with pytest.raises((ValueError, RuntimeError)):
        pf.parflex(C, [(1, 1), (1, 2), (2, 1)], [2, 3, 3], 0.1, L=10, profile_dir=None)


def test_workload_generator_deterministic():
    from parflexdtw_b200 import workloads as W
    a = W.make_pair(W.CONFIG0)
    b = W.make_pair(W.CONFIG0)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    assert a[0].shape == (12, 2000) and a[1].shape == (12, 2400)
    assert np.all(a[0] >= 0)
    C1 = W.cost_matrix_det(a[0][:, :50], a[1][:, :60])
    C2 = W.cost_matrix_host(a[0][:, :50], a[1][:, :60])
    assert np.max(np.abs(C1 - C2)) < 1e-14
