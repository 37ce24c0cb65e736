"""Device plan: one alignment's geometry and device workspace.

Thin owner of a ``pfx_plan*`` (include/parflexdtw_b200.h).  Device buffers
are exposed as zero-copy torch views through ``__cuda_array_interface__``.
torch supplies device memory for inputs and the current CUDA stream.
"""
from __future__ import annotations

import ctypes as ct
import weakref

import numpy as np
import torch

from . import _lib as L

_DT = {"f64": ("<f8", torch.float64, 8), "f32": ("<f4", torch.float32, 4),
       "i32": ("<i4", torch.int32, 4), "bf16": ("<u2", torch.uint16, 2),
       "u32": ("<u4", torch.int32, 4), "u8": ("|u1", torch.uint8, 1),
       "i64": ("<i8", torch.int64, 8)}

_BUF_DTYPE = {"EDGE_D": "f64", "EDGE_P": "i32", "BACKPTR": "u32", "EDGE_CF": "f64",
              "VALID": "u8", "D_ARR": "f64", "L_ARR": "f64", "TOP_D": "f64",
              "TOP_L": "f64", "RIGHT_D": "f64", "RIGHT_L": "f64", "SEG_NORM": "f64",
              "SEG_META": "i64", "D_PROP": "f64", "L_PROP": "f64", "COST": "f64",
              "FEAT_BF16": "bf16"}


class _DevView:
    """Minimal ``__cuda_array_interface__`` exporter for a plan buffer."""

    def __init__(self, ptr, shape, typestr):
        self.__cuda_array_interface__ = {
            "shape": tuple(int(s) for s in shape), "typestr": typestr,
            "data": (int(ptr), False), "version": 2, "strides": None}


def current_stream_ptr():
    return ct.c_void_p(torch.cuda.current_stream().cuda_stream)


def normalize_steps(steps, weights):
    st = np.asarray(steps, dtype=np.int64).reshape(-1, 2)
    w = np.asarray(weights, dtype=np.float64).reshape(-1)
    if st.shape[0] != w.shape[0]:
        raise ValueError("steps and weights must have the same length")
    return st, w


def _free_plan(handle):
    if handle:
        L.load().pfx_plan_destroy(handle)


class Plan:
    """Geometry + device workspace for an N x M cost matrix with tile length L."""

    def __init__(self, N, M, Lb, steps, weights, precision="fp64"):
        lib = L.load()
        if precision not in ("fp64", "fp32"):
            raise ValueError("precision must be 'fp64' or 'fp32'")
        self.precision = precision
        if not torch.cuda.is_available():
            raise RuntimeError("parflexdtw_b200 needs a CUDA device")
        torch.cuda.init()
        st, w = normalize_steps(steps, weights)
        self.steps = st
        self.weights = w
        self.N, self.M, self.L = int(N), int(M), int(Lb)
        h = ct.c_void_p()
        L.check(lib.pfx_plan_create_ex(self.N, self.M, self.L,
                                       L.i64_array(st.reshape(-1)),
                                       L.f64_array(w), st.shape[0],
                                       L.PFX_FP32 if precision == "fp32" else L.PFX_FP64,
                                       ct.byref(h)))
        self._h = h
        self._fin = weakref.finalize(self, _free_plan, h)
        info = (ct.c_int64 * 8)()
        L.check(lib.pfx_plan_info(h, info))
        (self.n1, self.n2, _, self.hop, self.S, self.b_words, self.device_bytes,
         self.warps) = (int(x) for x in info)
        self.device = torch.cuda.current_device()

    @classmethod
    def borrow(cls, handle, owner, N, M, Lb, steps, weights):
        """A Plan over a handle owned by ``owner`` (a batch): not destroyed
        here, and ``owner`` stays alive while the Plan does."""
        self = cls.__new__(cls)
        self.precision = getattr(owner, "precision", "fp64")
        self.steps, self.weights = normalize_steps(steps, weights)
        self.N, self.M, self.L = int(N), int(M), int(Lb)
        self._h = handle
        self._owner = owner
        self._fin = weakref.finalize(self, lambda: None)
        info = (ct.c_int64 * 8)()
        L.check(L.load().pfx_plan_info(handle, info))
        (self.n1, self.n2, _, self.hop, self.S, self.b_words, self.device_bytes,
         self.warps) = (int(x) for x in info)
        self.device = owner.device
        return self

    @property
    def handle(self):
        return self._h

    def close(self):
        self._fin()

    # -- zero-copy device views ------------------------------------------
    def view(self, name) -> torch.Tensor:
        lib = L.load()
        ptr, nb = ct.c_void_p(), ct.c_int64()
        L.check(lib.pfx_plan_buffer(self._h, L.BUF[name], ct.byref(ptr), ct.byref(nb)))
        kind = _BUF_DTYPE[name]
        if name == "COST" and self.precision == "fp32":
            kind = "f32"
        typestr, tdt, size = _DT[kind]
        n = nb.value // size
        shape = (n,)
        s4 = (self.n1, self.n2, 2, self.L)
        if name in ("EDGE_D", "EDGE_P", "EDGE_CF", "VALID", "D_ARR", "L_ARR", "D_PROP",
                    "L_PROP"):
            shape = s4
        elif name == "SEG_NORM":
            shape = (2, n // 2)
        elif name == "SEG_META":
            shape = (2, n // 12, 6)
        elif name == "FEAT_BF16":
            shape = (self.N + self.M, n // (self.N + self.M))
        t = torch.as_tensor(_DevView(ptr.value, shape, typestr),
                            device=f"cuda:{self.device}")
        if kind == "bf16":
            t = t.view(torch.bfloat16)
        t._pfx_owner = self  # keep the plan alive while the view lives
        return t

    def host(self, name) -> np.ndarray:
        return self.view(name).cpu().numpy()

    def cost_matrix(self) -> np.ndarray:
        """The loaded cost as an N x M host array, read back from the
        tile-skewed slabs (FP64, or FP32 in the FP32 form)."""
        if getattr(self, "tile_range", None):
            raise ValueError("a plan with a tile range holds part of the cost only")
        slab = self.host("COST")
        spanL = -(-(self.L + 63) // 16) * 16
        nSL = -(-self.L // 64)
        stride = nSL * spanL * 64
        out = np.zeros((self.N, self.M), dtype=slab.dtype)
        for t in range(self.n1 * self.n2):
            i, j = divmod(t, self.n2)
            r0, c0 = i * self.hop, j * self.hop
            R, W = min(self.L, self.N - r0), min(self.L, self.M - c0)
            span = -(-(W + 63) // 16) * 16
            nS = -(-R // 64)
            sl = slab[t * stride:t * stride + nS * span * 64].reshape(nS, span, 64)
            r = np.arange(R)
            k, rho = r // 64, r % 64
            c = np.arange(W)
            out[r0:r0 + R, c0:c0 + W] = sl[k[:, None], c[None, :] + rho[:, None], rho[:, None]]
        return out

    # -- cost loading ----------------------------------------------------
    def load_cost(self, C_dev: torch.Tensor, stream=None):
        """Copy a row-major cost matrix into the plan's tile-skewed layout
        (FP64; an FP32 plan also takes an FP32 matrix, and rounds an FP64
        one to FP32)."""
        if C_dev.stride(1) != 1:
            raise ValueError("cost matrix rows must be contiguous")
        lib = L.load()
        s = stream or current_stream_ptr()
        if C_dev.dtype == torch.float32:
            L.check(lib.pfx_plan_load_cost_f32(self._h, ct.c_void_p(C_dev.data_ptr()),
                                               C_dev.stride(0), s))
        elif C_dev.dtype == torch.float64:
            L.check(lib.pfx_plan_load_cost(self._h, ct.c_void_p(C_dev.data_ptr()),
                                           C_dev.stride(0), s))
        else:
            raise ValueError(f"cost matrix dtype {C_dev.dtype}: float64 or float32")

    def load_features(self, F1_dev: torch.Tensor, F2_dev: torch.Tensor, stream=None):
        """Build the cost 1 - L2norm(F1)^T L2norm(F2) straight into the plan's
        tile-skewed layout (F1: d x N, F2: d x M, FP64, contiguous).  FP32
        plans build it on the tensor cores from bf16 features."""
        for F, n in ((F1_dev, self.N), (F2_dev, self.M)):
            if F.dim() != 2 or F.shape[1] != n or F.dtype != torch.float64 or \
                    not F.is_contiguous() or not F.is_cuda:
                raise ValueError(f"features must be contiguous FP64 CUDA tensors of shape "
                                 f"(d, {n}); got {tuple(F.shape)} {F.dtype}")
        if F1_dev.shape[0] != F2_dev.shape[0]:
            raise ValueError("features must share the feature dimension")
        fn = L.load().pfx_plan_load_features_bf16 if self.precision == "fp32" else \
            L.load().pfx_plan_load_features
        L.check(fn(
            self._h, ct.c_void_p(F1_dev.data_ptr()), ct.c_void_p(F2_dev.data_ptr()),
            int(F1_dev.shape[0]), stream or current_stream_ptr()))

    def set_warps(self, nw):
        """Stage-1 warps per tile CTA (4, 8 or 16)."""
        L.check(L.load().pfx_plan_set_warps(self._h, int(nw)))
        self.warps = int(nw)

    def set_tile_mask(self, mask=None, stream=None):
        """Restrict cost building and stage 1 to the tiles set in ``mask``
        ((n1, n2) bool/uint8, host array or CUDA tensor); None lifts it."""
        lib = L.load()
        s = stream or current_stream_ptr()
        if mask is None:
            L.check(lib.pfx_plan_set_tile_mask(self._h, None, 0, s))
            return
        if isinstance(mask, torch.Tensor) and mask.is_cuda:
            m = mask.to(torch.uint8).contiguous()
            if m.numel() != self.n1 * self.n2:
                raise ValueError("mask must have n1 * n2 entries")
            L.check(lib.pfx_plan_set_tile_mask(self._h, ct.c_void_p(m.data_ptr()), 1, s))
            self._mask_keep = m
        else:
            m = np.ascontiguousarray(np.asarray(mask, dtype=np.uint8).reshape(-1))
            if m.size != self.n1 * self.n2:
                raise ValueError("mask must have n1 * n2 entries")
            L.check(lib.pfx_plan_set_tile_mask(self._h, m.ctypes.data_as(ct.c_void_p), 0, s))

    def set_tile_range(self, lo, hi, stream=None):
        """Hold cost slabs for tiles [lo, hi) of the tile order only and run
        stage 1 on them alone, for good (before any cost is loaded)."""
        L.check(L.load().pfx_plan_set_tile_range(self._h, int(lo), int(hi),
                                                 stream or current_stream_ptr()))
        self.tile_range = (int(lo), int(hi))

    # -- stages ----------------------------------------------------------
    @staticmethod
    def _cptr(C_dev):
        if C_dev is None:
            return ct.c_void_p(0), 0
        return ct.c_void_p(C_dev.data_ptr()), C_dev.stride(0)

    def stage1(self, C_dev: torch.Tensor = None, stream=None):
        """Stage 1; with ``C_dev`` it is loaded first, else the loaded cost is used."""
        p, ld = self._cptr(C_dev)
        L.check(L.load().pfx_stage1(self._h, p, ld, stream or current_stream_ptr()))

    def propagate(self, C_dev: torch.Tensor = None, stream=None, snapshot=False):
        lib = L.load()
        s = stream or current_stream_ptr()
        p, ld = self._cptr(C_dev)
        L.check(lib.pfx_stage2_propagate(self._h, p, ld, s))
        if snapshot:
            L.check(lib.pfx_snapshot_prop(self._h, s))

    def edges(self, C_dev: torch.Tensor = None, stream=None):
        """First part of ``propagate``: edge tensors and valid mask (the only
        stage-2 step that reads the cost)."""
        p, ld = self._cptr(C_dev)
        L.check(L.load().pfx_stage2_edges(self._h, p, ld, stream or current_stream_ptr()))

    def prop(self, stream=None):
        """Second part of ``propagate``: the cross-tile propagation."""
        L.check(L.load().pfx_stage2_prop(self._h, stream or current_stream_ptr()))

    def chain(self, start=None, stream=None) -> np.ndarray:
        """Tiles the stitched backtrace crosses, end tile first, as an (n, 2)
        int array of (i, j); reads no backpointers.  Synchronises."""
        lib = L.load()
        s = stream or current_stream_ptr()
        buf = (ct.c_int32 * 202)()
        n = ct.c_int32()
        fb, (i, j, e, x) = (1, (0, 0, 0, 0)) if start is None else (0, start)
        L.check(lib.pfx_stage2_chain(self._h, fb, int(i), int(j), int(e), int(x), buf, 101,
                                     ct.byref(n), s))
        return np.frombuffer(buf, dtype=np.int32)[:2 * n.value].reshape(-1, 2).copy()

    def scan(self, beta, stream=None):
        L.check(L.load().pfx_stage2_scan(self._h, float(beta),
                                         stream or current_stream_ptr()))

    def stitch(self, start=None, stream=None):
        lib = L.load()
        s = stream or current_stream_ptr()
        if start is None:
            L.check(lib.pfx_stage2_stitch(self._h, 1, 0, 0, 0, 0, s))
        else:
            i, j, e, x = (int(v) for v in start)
            L.check(lib.pfx_stage2_stitch(self._h, 0, i, j, e, x, s))

    def run(self, C_dev: torch.Tensor = None, beta=0.1, stream=None):
        p, ld = self._cptr(C_dev)
        L.check(L.load().pfx_parflex_device(self._h, p, ld, float(beta),
                                            stream or current_stream_ptr()))

    def result(self, stream=None, raise_no_endpoint=True):
        """(best_cost, best_end[6], found, path_len); synchronises the stream."""
        lib = L.load()
        b = ct.c_double()
        e = (ct.c_int64 * 7)()
        n = ct.c_int64()
        st = lib.pfx_result(self._h, stream or current_stream_ptr(), ct.byref(b), e,
                            ct.byref(n))
        if st != L.PFX_ERR_NO_ENDPOINT or raise_no_endpoint:
            L.check(st)
        return b.value, tuple(int(x) for x in e[:6]), bool(e[6]), n.value

    def path(self, n, stream=None) -> np.ndarray:
        """The last stitched path as a (K, 2) int64 array, start first."""
        out = np.empty((max(int(n), 1), 2), dtype=np.int64)
        L.check(L.load().pfx_copy_path(self._h, stream or current_stream_ptr(),
                                       out.ctypes.data_as(ct.POINTER(ct.c_int64)),
                                       out.shape[0]))
        return out[:n]
