"""pfx_flexdtw_tile_noalloc against pfx_flexdtw_tile, through the C ABI.

The no-allocation variant exists for callers that cannot call cudaMalloc: an
online aligner that runs the tile DP on every incoming block of audio frames
and must not block on the allocator (or on the device-wide synchronisation
cudaMalloc / cudaFree can cause), and host applications that reserve all
device memory themselves and forbid libraries from allocating.  It keeps the
kernel's scratch in a fixed device array of the library instead, so its
results must be identical to the allocating entry point's -- bit for bit, the
tolerance every parity test here uses -- on consecutive calls that reuse that
array.

This file is collected last on purpose, and passes both alone in a fresh
process (where its first call also sets the scratch up) and after the rest of
the suite.
"""
import ctypes as ct

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - CPU container
    pytest.skip("needs a CUDA device", allow_module_level=True)

from parflexdtw_b200 import _lib  # noqa: E402

STEPS = (ct.c_int64 * 6)(1, 1, 1, 2, 2, 1)
WEIGHTS = (ct.c_double * 3)(2.0, 3.0, 3.0)


def _run(fn, Cd, r0, r1, c0, c1):
    R, W = r1 - r0, c1 - c0
    D = torch.empty((R, W), dtype=torch.float64, device="cuda")
    P = torch.empty((R, W), dtype=torch.int32, device="cuda")
    B = torch.empty((R, W), dtype=torch.int8, device="cuda")
    base = Cd.data_ptr() + (r0 * Cd.stride(0) + c0) * 8
    stream = ct.c_void_p(torch.cuda.current_stream().cuda_stream)
    st = fn(base, Cd.stride(0), R, W, STEPS, WEIGHTS, 3, D.data_ptr(), P.data_ptr(),
            B.data_ptr(), stream)
    assert st == _lib.PFX_OK, _lib.load().pfx_last_error()
    torch.cuda.synchronize()
    return D.cpu().numpy(), P.cpu().numpy(), B.cpu().numpy()


def test_noalloc_matches_allocating_entry_point_on_consecutive_calls():
    lib = _lib.load()
    rng = np.random.RandomState(1234)
    C = np.abs(rng.randn(2600, 2300)) * 0.2
    Cd = torch.from_numpy(C).cuda()
    tiles = [(0, 2048, 0, 2048), (513, 1800, 77, 1111)]
    expect = [_run(lib.pfx_flexdtw_tile, Cd, *t) for t in tiles]
    # two no-allocation calls in a row, the second reusing the first's scratch
    got = [_run(lib.pfx_flexdtw_tile_noalloc, Cd, *t) for t in tiles]
    for (De, Pe, Be), (Dg, Pg, Bg) in zip(expect, got):
        assert np.array_equal(De, Dg)
        assert np.array_equal(Pe, Pg)
        assert np.array_equal(Be, Bg)


def test_noalloc_rejects_tiles_beyond_its_scratch():
    lib = _lib.load()
    Cd = torch.zeros((4, 2049), dtype=torch.float64, device="cuda")
    out = torch.empty((4, 2049), dtype=torch.float64, device="cuda")
    st = lib.pfx_flexdtw_tile_noalloc(Cd.data_ptr(), 2049, 4, 2049, STEPS, WEIGHTS, 3,
                                      out.data_ptr(), out.data_ptr(), out.data_ptr(),
                                      ct.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == _lib.PFX_ERR_TOO_LARGE
    assert b"2048" in lib.pfx_last_error()
