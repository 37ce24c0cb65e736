"""pfx_flexdtw_tile_noalloc against pfx_flexdtw_tile and the golden tiles,
through the C ABI.

The no-allocation variant exists for callers that cannot call cudaMalloc: an
online aligner that runs the tile DP on every incoming block of audio frames
and must not block on the allocator (or on the device-wide synchronisation
cudaMalloc / cudaFree can cause), and host applications that reserve all
device memory themselves and forbid libraries from allocating.  It keeps the
kernel's scratch in a fixed device array of the library instead, so its
results must be identical to the allocating entry point's -- bit for bit, the
tolerance every parity test here uses -- on consecutive calls that reuse that
array, and identical to the reference's own outputs on the golden tiles.

This file is collected last on purpose, and passes both alone in a fresh
process (where its first call also sets the scratch up) and after the rest of
the suite.
"""
import ctypes as ct

import numpy as np
import pytest

from golden_util import load, names

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - CPU container
    pytest.skip("needs a CUDA device", allow_module_level=True)

from parflexdtw_b200 import _lib  # noqa: E402

STD = ((1, 1), (1, 2), (2, 1))
STD_W = (2.0, 3.0, 3.0)


def _steps(steps, weights):
    st = np.asarray(steps, dtype=np.int64).reshape(-1)
    w = np.asarray(weights, dtype=np.float64).reshape(-1)
    return (ct.c_int64 * st.size)(*st.tolist()), (ct.c_double * w.size)(*w.tolist()), w.size


def _run(fn, Cd, r0, r1, c0, c1, steps=STD, weights=STD_W):
    R, W = r1 - r0, c1 - c0
    D = torch.empty((R, W), dtype=torch.float64, device="cuda")
    P = torch.empty((R, W), dtype=torch.int32, device="cuda")
    B = torch.empty((R, W), dtype=torch.int8, device="cuda")
    base = Cd.data_ptr() + (r0 * Cd.stride(0) + c0) * 8
    stream = ct.c_void_p(torch.cuda.current_stream().cuda_stream)
    st, w, n = _steps(steps, weights)
    status = fn(base, Cd.stride(0), R, W, st, w, n, D.data_ptr(), P.data_ptr(), B.data_ptr(),
                stream)
    assert status == _lib.PFX_OK, _lib.load().pfx_last_error()
    torch.cuda.synchronize()
    return D.cpu().numpy(), P.cpu().numpy(), B.cpu().numpy()


def _same(a, b):
    return all(np.array_equal(x, y) for x, y in zip(a, b))


def test_noalloc_matches_allocating_entry_point_on_consecutive_calls():
    lib = _lib.load()
    rng = np.random.RandomState(1234)
    C = np.abs(rng.randn(2600, 2300)) * 0.2
    Cd = torch.from_numpy(C).cuda()
    tiles = [(0, 2048, 0, 2048), (513, 1800, 77, 1111)]
    expect = [_run(lib.pfx_flexdtw_tile, Cd, *t) for t in tiles]
    # two no-allocation calls in a row, the second reusing the first's scratch
    got = [_run(lib.pfx_flexdtw_tile_noalloc, Cd, *t) for t in tiles]
    for e, g in zip(expect, got):
        assert _same(e, g)


@pytest.mark.parametrize("name", names("tile"))
def test_noalloc_matches_golden_tiles(name):
    """Straight against the reference's own FlexDTW.flexdtw outputs (D, P, B),
    twice in a row on the same scratch."""
    g = load("tile", name)
    C = np.ascontiguousarray(g["C"])
    Cd = torch.from_numpy(C).cuda()
    fn = _lib.load().pfx_flexdtw_tile_noalloc
    for _ in range(2):
        D, P, B = _run(fn, Cd, 0, C.shape[0], 0, C.shape[1], g["steps"], g["weights"])
        assert np.array_equal(D, g["D"])
        assert np.array_equal(P, g["P"])
        assert np.array_equal(B, g["B"])


@pytest.mark.parametrize("steps,weights", [(((1, 1), (2, 1)), (2.0, 3.0)),
                                           (((2, 1), (1, 1), (1, 2)), (3.0, 1.5, 3.0))])
@pytest.mark.parametrize("tile", [(0, 1, 0, 700), (0, 900, 5, 6), (3, 260, 11, 1800),
                                  (100, 2000, 0, 37)])
def test_noalloc_other_steps_and_thin_tiles(steps, weights, tile):
    """The generic-step kernel and the one-row / one-column branch."""
    lib = _lib.load()
    rng = np.random.RandomState(99)
    C = np.abs(rng.randn(2100, 1900)) * 0.3
    Cd = torch.from_numpy(C).cuda()
    expect = _run(lib.pfx_flexdtw_tile, Cd, *tile, steps, weights)
    got = [_run(lib.pfx_flexdtw_tile_noalloc, Cd, *tile, steps, weights) for _ in range(2)]
    for g in got:
        assert _same(expect, g)


def _cudart():
    # the CUDA runtime the library itself is linked against (already loaded)
    _lib.load()
    return ct.CDLL("libcudart.so.12")


def _pool_used_high(rt, pool):
    v = ct.c_uint64(0)
    assert rt.cudaMemPoolGetAttribute(pool, 8, ct.byref(v)) == 0  # UsedMemHigh
    return v.value


def _reset_pool_high(rt, pool):
    z = ct.c_uint64(0)
    assert rt.cudaMemPoolSetAttribute(pool, 8, ct.byref(z)) == 0


def test_noalloc_allocates_no_device_memory():
    """Neither the device's default memory pool (which the allocating entry
    point draws its scratch from, so the probe is shown to see it) nor the
    device's free memory moves during no-allocation calls."""
    lib = _lib.load()
    rt = _cudart()
    rt.cudaDeviceGetDefaultMemPool.argtypes = [ct.POINTER(ct.c_void_p), ct.c_int]
    rt.cudaMemPoolGetAttribute.argtypes = [ct.c_void_p, ct.c_int, ct.c_void_p]
    rt.cudaMemPoolSetAttribute.argtypes = [ct.c_void_p, ct.c_int, ct.c_void_p]
    rt.cudaMemGetInfo.argtypes = [ct.POINTER(ct.c_size_t), ct.POINTER(ct.c_size_t)]
    pool = ct.c_void_p()
    assert rt.cudaDeviceGetDefaultMemPool(ct.byref(pool), torch.cuda.current_device()) == 0
    rng = np.random.RandomState(5)
    C = np.abs(rng.randn(1500, 1700)) * 0.2
    Cd = torch.from_numpy(C).cuda()
    # every output tensor the calls below need, allocated before the probe
    outs = [(torch.empty((1500, 1700), dtype=torch.float64, device="cuda"),
             torch.empty((1500, 1700), dtype=torch.int32, device="cuda"),
             torch.empty((1500, 1700), dtype=torch.int8, device="cuda")) for _ in range(3)]
    st, w, n = _steps(STD, STD_W)
    stream = ct.c_void_p(torch.cuda.current_stream().cuda_stream)

    def call(fn, o):
        s = fn(Cd.data_ptr(), Cd.stride(0), 1500, 1700, st, w, n, o[0].data_ptr(),
               o[1].data_ptr(), o[2].data_ptr(), stream)
        assert s == _lib.PFX_OK, lib.pfx_last_error()
        torch.cuda.synchronize()

    call(lib.pfx_flexdtw_tile_noalloc, outs[0])  # scratch address set up
    free0, total = ct.c_size_t(), ct.c_size_t()
    _reset_pool_high(rt, pool)
    base = _pool_used_high(rt, pool)
    assert rt.cudaMemGetInfo(ct.byref(free0), ct.byref(total)) == 0
    call(lib.pfx_flexdtw_tile_noalloc, outs[1])
    call(lib.pfx_flexdtw_tile_noalloc, outs[2])
    free1 = ct.c_size_t()
    assert rt.cudaMemGetInfo(ct.byref(free1), ct.byref(total)) == 0
    assert _pool_used_high(rt, pool) == base
    assert free1.value == free0.value
    # the probe does see the allocating entry point's scratch
    call(lib.pfx_flexdtw_tile, outs[1])
    assert _pool_used_high(rt, pool) > base
    for o in outs[1:]:
        assert torch.equal(o[0], outs[0][0]) and torch.equal(o[1], outs[0][1])
        assert torch.equal(o[2], outs[0][2])


def test_noalloc_rejects_tiles_beyond_its_scratch():
    lib = _lib.load()
    Cd = torch.zeros((4, 2049), dtype=torch.float64, device="cuda")
    out = torch.empty((4, 2049), dtype=torch.float64, device="cuda")
    st, w, n = _steps(STD, STD_W)
    status = lib.pfx_flexdtw_tile_noalloc(Cd.data_ptr(), 2049, 4, 2049, st, w, n,
                                          out.data_ptr(), out.data_ptr(), out.data_ptr(),
                                          ct.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert status == _lib.PFX_ERR_TOO_LARGE
    assert b"2048" in lib.pfx_last_error()
