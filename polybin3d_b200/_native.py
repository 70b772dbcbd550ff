"""ctypes binding of the C ABI (include/polybin3d_b200.h) on torch device tensors.

Torch supplies device memory and the current CUDA stream; every computation is a call
into libpb_b200.so.  There is no fallback: if the library or a CUDA device is missing,
loading raises.
"""
import ctypes
import os
import threading

import numpy as np
import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libpb_b200.so")

PB_F32, PB_F64 = 0, 1
PB_F32_SRC_F64 = 2  # shell_synth only: FP32 maps from a complex128 source
PB_FFT_R2C, PB_FFT_C2R = 0, 1
PB_RED_ABS2, PB_RED_CROSS, PB_RED_REAL2 = 0, 1, 2
PB_TRIPLET_SIMT, PB_TRIPLET_TC = 0, 1
PB_EW_MUL, PB_EW_PRODDIFF, PB_EW_WIDEN = 0, 1, 2
FILTER_MAX_MAPS = 128
SYNTH_MAX_MAPS = 64
SYNTH_WS_BYTES = 8 << 30  # transform workspace per pb_shell_synth call

_ERRORS = {-1: ValueError, -2: RuntimeError, -3: RuntimeError, -4: MemoryError, -5: NotImplementedError,
           -6: TimeoutError}


PB_GRID_LOS = 1


class PBGrid(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int32 * 3), ("flags", ctypes.c_int32), ("kf", ctypes.c_double * 3),
                ("los", ctypes.c_double * 3)]


class PBTuning(ctypes.Structure):
    _fields_ = [("tc_tile", ctypes.c_int32), ("tc_stages", ctypes.c_int32), ("tc_chain", ctypes.c_int32),
                ("red_method", ctypes.c_int32), ("red_warps", ctypes.c_int32), ("red_waves", ctypes.c_int32),
                ("tc_wait", ctypes.c_int32), ("tc_dsets", ctypes.c_int32)]


TUNING_FIELDS = [f for f, _ in PBTuning._fields_]

_lib = None
_lib_lock = threading.Lock()

_P = ctypes.c_void_p
_I = ctypes.c_int
_I64 = ctypes.c_int64
_D = ctypes.c_double
_SZ = ctypes.c_size_t
_GP = ctypes.POINTER(PBGrid)

SIGNATURES = {
    "pb_abi_version": ([], _I),
    "pb_last_error": ([], ctypes.c_char_p),
    "pb_fft_plan_create": ([_GP, _I, _I, _I, ctypes.POINTER(_P), ctypes.POINTER(_SZ)], _I),
    "pb_fft_exec": ([_P, _P, _P, _P, _P], _I),
    "pb_fft_plan_destroy": ([_P], _I),
    "pb_spectral_filter": ([_GP, _P, _I, _P, _I64, _P, _I, _P, _P, _P, _P, _P, _P, _P, _P, _P, _I, _P], _I),
    "pb_binned_filter": ([_GP, _I, _P, _P, _P, _I, _P, _I, _P, _P, _I, _D, _P], _I),
    "pb_bilinear_plan": ([_I, _I, _P, _P, _P, _P, _I, _P, ctypes.POINTER(_SZ), _P], _I),
    "pb_bilinear_maps": ([_I, _I64, _P, _I, _P, _I, _I, _P, _P], _I),
    "pb_shell_synth_workspace_size": ([_GP, _P, _I, _I, _P, ctypes.POINTER(_SZ)], _I),
    "pb_shell_synth": ([_GP, _P, _I, _P, _I64, _I, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _SZ, _P], _I),
    "pb_bin_reduce_workspace_size": ([_GP, _I, _I, _I, ctypes.POINTER(_SZ)], _I),
    "pb_bin_reduce": ([_GP, _I, _I, _P, _P, _I, _I64, _P, _I, _P, _I, _D, _P, _I, _P, _SZ, _P], _I),
    "pb_bin_reduce_noalloc": ([_GP, _I, _I, _P, _P, _I, _I64, _P, _I, _P, _I, _D, _P, _I, _P], _I),
    "pb_set_tuning": ([ctypes.POINTER(PBTuning)], _I),
    "pb_get_tuning": ([ctypes.POINTER(PBTuning)], _I),
    "pb_triplet_plan": ([_I, _I, _I, _P, _I, _P, ctypes.POINTER(_SZ), _P], _I),
    "pb_triplet_workspace_size": ([_I, _I, _I64, _P, _I, ctypes.POINTER(_SZ)], _I),
    "pb_triplet_contract": ([_I, _I, _P, _I, _P, _I, _P, _I, _I64, _P, _P, _D, _P, _P, _SZ, _P], _I),
    "pb_tiled_maps_bytes": ([_I, _I, _I64, ctypes.POINTER(_SZ)], _I),
    "pb_tile_maps": ([_P, _I, _I, _I64, _P, _P], _I),
    "pb_triplet_contract_tiled": ([_I, _P, _I, _I, _I64, _P, _P, _D, _P, _P, _SZ, _P], _I),
    "pb_shell_synth_tiled": ([_GP, _P, _I, _P, _I64, _I, _I, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _SZ, _P], _I),
    "pb_elementwise": ([_I, _I, _I64, _P, _P, _I64, _P, _P, _D, _P, _P], _I),
    "pb_grf_from_noise": ([_GP, _I, _P, _P, _I, _P, _D, _P, _P], _I),
    "pb_grf_philox": ([_GP, _I, _P, _I, _P, _D, _P, _P], _I),
    "pb_pair_products": ([_I, _I64, _P, _P, _P, _P, _P, _I, _D, _P, _P], _I),
    "pb_shell_rows_workspace_size": ([_I64, _I, _I, ctypes.POINTER(_SZ)], _I),
    "pb_shell_rows": ([_GP, _I, _P, _I, _P, _I, _P, _I64, _P, _P, _I, _D, _P, _I64, _P, _SZ, _P], _I),
}


def load(path=LIB_PATH):
    """Load libpb_b200.so (raises if absent: there is no CPU fallback)."""
    global _lib
    with _lib_lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(path):
            raise ImportError("polybin3d_b200: CUDA extension %s is not built "
                              "(run `python -m polybin3d_b200.build`)" % path)
        lib = ctypes.CDLL(path)
        for name, (args, res) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = res
        if lib.pb_abi_version() != 2:
            raise ImportError("polybin3d_b200: ABI version mismatch")
        _lib = lib
        return lib


LAUNCHES = [0]  # kernels of this library launched through these wrappers (bench bookkeeping)


def _count(n):
    LAUNCHES[0] += n


def check(status, what=""):
    if status != 0:
        msg = load().pb_last_error().decode(errors="replace")
        raise _ERRORS.get(status, RuntimeError)("%s: %s" % (what, msg) if what else msg)


def require_cuda():
    if not torch.cuda.is_available():
        raise RuntimeError("polybin3d_b200 backend='cuda' needs a CUDA device; there is no CPU fallback")
    load()


def set_tuning(cfg=None):
    """Launch shapes for this host thread (pb_set_tuning): a dict of PBTuning fields, missing
    or zero fields meaning the built-in default; None restores every default."""
    if cfg is None:
        check(load().pb_set_tuning(None), "pb_set_tuning")
        return
    t = PBTuning(*[int(cfg.get(f, 0)) for f in TUNING_FIELDS])
    check(load().pb_set_tuning(ctypes.byref(t)), "pb_set_tuning")


def get_tuning():
    t = PBTuning()
    check(load().pb_get_tuning(ctypes.byref(t)), "pb_get_tuning")
    return {f: int(getattr(t, f)) for f in TUNING_FIELDS}


def stream_ptr():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def ptr(t):
    return ctypes.c_void_p(0 if t is None else t.data_ptr())


def hptr(a):
    """Host numpy array -> void*."""
    return ctypes.c_void_p(a.ctypes.data)


def precision_of(dtype):
    if dtype in (torch.float32, torch.complex64):
        return PB_F32
    if dtype in (torch.float64, torch.complex128):
        return PB_F64
    raise TypeError("unsupported dtype %s" % dtype)


# --------------------------------------------------------------------------------------
# workspace arena (torch-allocated scratch, reused across calls on the same stream)
# --------------------------------------------------------------------------------------
class Workspace:
    def __init__(self, device):
        self.device = device
        self.bufs = {}

    def get(self, nbytes, slot="default"):
        nbytes = max(int(nbytes), 256)
        b = self.bufs.get(slot)
        if b is None or b.numel() < nbytes:
            b = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
            self.bufs[slot] = b
        return b


# --------------------------------------------------------------------------------------
# FFT plans
# --------------------------------------------------------------------------------------
class FFTPlan:
    def __init__(self, grid, batch, precision, direction):
        lib = load()
        h = ctypes.c_void_p()
        ws = ctypes.c_size_t()
        check(lib.pb_fft_plan_create(ctypes.byref(grid), batch, precision, direction, ctypes.byref(h),
                                     ctypes.byref(ws)), "pb_fft_plan_create")
        self.h, self.ws_bytes = h, ws.value
        self.batch, self.precision, self.direction = batch, precision, direction

    def exec(self, inp, out, workspace):
        check(load().pb_fft_exec(self.h, ptr(inp), ptr(out), ptr(workspace), stream_ptr()), "pb_fft_exec")

    def __del__(self):
        try:
            if self.h:
                load().pb_fft_plan_destroy(self.h)
        except Exception:
            pass


# --------------------------------------------------------------------------------------
# kernels
# --------------------------------------------------------------------------------------
def spectral_filter(grid, precision, src, out, maps, w=None, accumulate=False, src_stride=None, out_n=None,
                    dst=None):
    """maps: list of (src_idx, lo, hi, l1, l2, scale, wpow) -> writes out[m] (torch, complex);
    out_n: output grid dims (same frequencies on another grid), None = the input grid;
    dst: output index per entry (outputs may repeat; needs accumulate)."""
    lib = load()
    on = None if out_n is None else np.ascontiguousarray(out_n, dtype=np.int32)
    n = len(maps)
    if n == 0:
        return
    for c0 in range(0, n, FILTER_MAX_MAPS):
        chunk = maps[c0:c0 + FILTER_MAX_MAPS]
        arr = np.asarray(chunk, dtype=np.float64)
        si = np.ascontiguousarray(arr[:, 0].astype(np.int32))
        lo = np.ascontiguousarray(arr[:, 1])
        hi = np.ascontiguousarray(arr[:, 2])
        l1 = np.ascontiguousarray(arr[:, 3].astype(np.int32))
        l2 = np.ascontiguousarray(arr[:, 4].astype(np.int32))
        sc = np.ascontiguousarray(arr[:, 5])
        wp = np.ascontiguousarray(arr[:, 6].astype(np.int32))
        if dst is None:
            o = out[c0:c0 + len(chunk)]
            di = None
        else:
            o = out
            di = np.ascontiguousarray(np.asarray(dst[c0:c0 + len(chunk)], dtype=np.int32))
        stride = src_stride if src_stride is not None else (src[0].numel() if src is not None and src.dim() == 4 else 0)
        check(lib.pb_spectral_filter(ctypes.byref(grid), None if on is None else hptr(on), precision, ptr(src),
                                     stride, ptr(o), len(chunk), hptr(si), None if di is None else hptr(di),
                                     hptr(lo), hptr(hi), hptr(l1), hptr(l2), hptr(sc), hptr(wp),
                                     ptr(w), int(bool(accumulate)), stream_ptr()), "pb_spectral_filter")
        _count(1)


def bin_reduce(grid, precision, mode, a, b, n_rows, edges, ells, scale, out, ws, accumulate=False, row_stride=0):
    lib = load()
    edges = np.ascontiguousarray(edges, dtype=np.float64)
    nk = len(edges) - 1
    ells = np.ascontiguousarray(np.asarray(ells, dtype=np.int32).reshape(-1))
    n_ell = len(ells) // 2
    nbytes = ctypes.c_size_t()
    check(lib.pb_bin_reduce_workspace_size(ctypes.byref(grid), n_rows, nk, n_ell, ctypes.byref(nbytes)),
          "pb_bin_reduce_workspace_size")
    buf = ws.get(nbytes.value, "binred")
    check(lib.pb_bin_reduce(ctypes.byref(grid), precision, mode, ptr(a), ptr(b), n_rows, row_stride, hptr(edges), nk,
                            hptr(ells), n_ell, scale, ptr(out), int(bool(accumulate)), ptr(buf), buf.numel(),
                            stream_ptr()), "pb_bin_reduce")
    _count(2)


def elementwise(op, x, y, z=None, u=None, s=1.0, out=None, y_period=0):
    """out = s*x*y (MUL, y read at i % y_period if y_period) or s*(x*y - z*u) (PRODDIFF)."""
    lib = load()
    out = torch.empty_like(x) if out is None else out
    check(lib.pb_elementwise(precision_of(x.dtype), op, x.numel(), ptr(x), ptr(y), int(y_period), ptr(z), ptr(u),
                             float(s), ptr(out), stream_ptr()), "pb_elementwise")
    _count(1)
    return out


def widen(x, out=None):
    """FP64 copy of an FP32 tensor (exact), by the library's vectorised kernel."""
    if x.dtype != torch.float32 or not x.is_contiguous():
        raise ValueError("widen: a contiguous float32 tensor")
    out = torch.empty(x.shape, dtype=torch.float64, device=x.device) if out is None else out
    check(load().pb_elementwise(PB_F32, PB_EW_WIDEN, x.numel(), ptr(x), None, 0, None, None, 0.0, ptr(out),
                                stream_ptr()), "pb_elementwise")
    _count(1)
    return out


def grf_philox(grid, precision, seeds, amp, scale, out):
    """Half-spectrum GRFs from on-device Philox noise; seeds: device int64 (n_batch,)."""
    check(load().pb_grf_philox(ctypes.byref(grid), precision, ptr(seeds), seeds.numel(), ptr(amp), float(scale),
                               ptr(out), stream_ptr()), "pb_grf_philox")
    _count(1)
    return out


def grf_from_noise(grid, precision, noise_re, noise_im, amp, scale, out):
    lib = load()
    nb = noise_re.shape[0] if noise_re.dim() == 4 else 1
    check(lib.pb_grf_from_noise(ctypes.byref(grid), precision, ptr(noise_re), ptr(noise_im), nb, ptr(amp),
                                float(scale), ptr(out), stream_ptr()), "pb_grf_from_noise")
    _count(1)
    return out


class TripletPlan:
    """Device work-item table for a fixed triplet list (pb_triplet_plan)."""

    def __init__(self, n_a, n_b, n_c, idx, device):
        lib = load()
        idx = np.ascontiguousarray(np.asarray(idx, dtype=np.int32).reshape(-1, 3))
        self.n_a, self.n_b, self.n_c, self.n_trip = n_a, n_b, n_c, len(idx)
        nbytes = ctypes.c_size_t()
        self.counts = np.zeros(4, dtype=np.int32)
        check(lib.pb_triplet_plan(n_a, n_b, n_c, hptr(idx), len(idx), None, ctypes.byref(nbytes),
                                  hptr(self.counts)), "pb_triplet_plan")
        host = np.zeros(nbytes.value, dtype=np.uint8)
        check(lib.pb_triplet_plan(n_a, n_b, n_c, hptr(idx), len(idx), hptr(host), ctypes.byref(nbytes),
                                  hptr(self.counts)), "pb_triplet_plan")
        self.host_table = host
        self.n_items, self.n_pairs = int(self.counts[0]), int(self.counts[1])
        self.factor_max = int(idx[:, :2].max()) if len(idx) else -1
        self.table = torch.from_numpy(host).to(device)

    def workspace_bytes(self, precision, method, n_vox):
        nbytes = ctypes.c_size_t()
        check(load().pb_triplet_workspace_size(precision, method, n_vox, hptr(self.counts), self.n_c,
                                               ctypes.byref(nbytes)), "pb_triplet_workspace_size")
        return nbytes.value

    def contract(self, A, B, C, out, ws, method=PB_TRIPLET_SIMT, scale=1.0):
        """A, B, C: torch (n_maps, ...) real maps of one precision; out: float64 device (n_trip,)."""
        prec = precision_of(A.dtype)
        n_vox = A[0].numel()
        buf = ws.get(self.workspace_bytes(prec, method, n_vox), "triplet")
        check(load().pb_triplet_contract(prec, method, ptr(A), A.shape[0], ptr(B), B.shape[0], ptr(C), C.shape[0],
                                         n_vox, ptr(self.table), hptr(self.counts), float(scale), ptr(out),
                                         ptr(buf), buf.numel(), stream_ptr()), "pb_triplet_contract")
        _count(2)
        return out

    def contract_tiled(self, tiled, out, ws, method=PB_TRIPLET_TC, scale=1.0):
        """The contraction with A = B = C = a TiledMaps set (plan made for n_a = n_b = n_c = its
        maps, pair factors among its first n_factor maps)."""
        if not (self.n_a == self.n_b == self.n_c == tiled.n_maps) or self.factor_max >= tiled.n_factor:
            raise ValueError("contract_tiled: the plan (%d/%d/%d maps, pair factors up to %d) does not fit a set of "
                             "%d maps with %d factor maps" % (self.n_a, self.n_b, self.n_c, self.factor_max,
                                                               tiled.n_maps, tiled.n_factor))
        buf = ws.get(self.workspace_bytes(PB_F32, method, tiled.n_vox), "triplet")
        check(load().pb_triplet_contract_tiled(method, ptr(tiled.data), tiled.n_maps, tiled.n_factor, tiled.n_vox,
                                               ptr(self.table), hptr(self.counts), float(scale), ptr(out), ptr(buf),
                                               buf.numel(), stream_ptr()), "pb_triplet_contract_tiled")
        _count(2)
        return out


def tiled_maps_bytes(n_maps, n_factor, n_vox):
    nbytes = ctypes.c_size_t()
    check(load().pb_tiled_maps_bytes(int(n_maps), int(n_factor), int(n_vox), ctypes.byref(nbytes)),
          "pb_tiled_maps_bytes")
    return nbytes.value


def _tiled_dims(n_maps, n_factor):
    F, P = (n_factor + 7) // 8 * 8, (n_maps + 15) // 16 * 16
    return F, P, 512 * (F + P)


def tiled_factor_offsets(n_maps, n_factor, n_vox):
    """Host int64 [n_factor, n_vox]: byte offset of each voxel of each factor map (FP32)."""
    F, P, tb = _tiled_dims(n_maps, n_factor)
    v = np.arange(n_vox, dtype=np.int64)[None, :]
    m = np.arange(n_factor, dtype=np.int64)[:, None]
    w = v & 127
    return (v >> 7) * tb + ((w >> 5) * F + m) * 128 + ((((w & 31) >> 2) ^ (m & 7)) << 4) + (w & 3) * 4


def tiled_c_offsets(n_maps, n_factor, n_vox):
    """Host int64 [2, n_maps, n_vox]: byte offsets of the bf16 hi (0) and lo (1) parts."""
    F, P, tb = _tiled_dims(n_maps, n_factor)
    v = np.arange(n_vox, dtype=np.int64)[None, None, :]
    r = np.arange(n_maps, dtype=np.int64)[None, :, None] + np.asarray([0, P], dtype=np.int64)[:, None, None]
    w = v & 127
    return ((v >> 7) * tb + 512 * F + (w >> 4) * 64 * P + (r >> 3) * 256 + (r & 7) * 32 +
            ((((w & 15) >> 3) ^ ((r >> 2) & 1)) << 4) + (w & 7) * 2)


class TiledMaps:
    """A tiled map set (include/polybin3d_b200.h): n_maps f32 maps on `shape`, the first
    n_factor kept in FP32 as pair factors and every map split into bf16 hi + lo parts, per
    tile of 128 voxels in the tensor-core contraction's staging layout.  data: uint8 bytes."""

    def __init__(self, n_maps, n_factor, shape, device, data=None):
        self.n_maps, self.n_factor, self.shape = int(n_maps), int(n_factor), tuple(int(n) for n in shape)
        self.n_vox = int(np.prod(self.shape))
        n = tiled_maps_bytes(self.n_maps, self.n_factor, self.n_vox)
        self.data = torch.empty(n, dtype=torch.uint8, device=device) if data is None else data
        if self.data.numel() < n or self.data.dtype != torch.uint8:
            raise ValueError("TiledMaps: data must hold %d bytes" % n)

    @classmethod
    def from_maps(cls, maps, n_factor):
        """Tile (n_maps, *shape) float32 device maps (pb_tile_maps)."""
        maps = maps.contiguous()
        t = cls(maps.shape[0], n_factor, maps.shape[1:], maps.device)
        check(load().pb_tile_maps(ptr(maps), t.n_maps, t.n_factor, t.n_vox, ptr(t.data), stream_ptr()),
              "pb_tile_maps")
        _count(1)
        return t

    def factor_maps(self):
        """(n_factor, *shape) float32: the FP32 factor maps (a device gather)."""
        off = torch.as_tensor(tiled_factor_offsets(self.n_maps, self.n_factor, self.n_vox) // 4, device=self.data.device)
        return self.data.view(torch.float32)[off].reshape((self.n_factor,) + self.shape)

    def split_parts(self):
        """(hi, lo): (n_maps, *shape) bfloat16 parts of every map (a device gather)."""
        off = torch.as_tensor(tiled_c_offsets(self.n_maps, self.n_factor, self.n_vox) // 2, device=self.data.device)
        x = self.data.view(torch.bfloat16)[off]
        return x[0].reshape((self.n_maps,) + self.shape), x[1].reshape((self.n_maps,) + self.shape)


def pair_products(X, Y, pairs, Z=None, U=None, s=1.0, out=None):
    """out[p] = s*(X[i]Y[j] - Z[i]U[j]) for host (i, j) pairs; X.. are (n, ...) real maps."""
    pairs = np.ascontiguousarray(np.asarray(pairs, dtype=np.int32).reshape(-1, 2))
    n_vox = X[0].numel()
    if out is None:
        out = torch.empty((len(pairs),) + tuple(X.shape[1:]), dtype=X.dtype, device=X.device)
    check(load().pb_pair_products(precision_of(X.dtype), n_vox, ptr(X), ptr(Y), ptr(Z), ptr(U), hptr(pairs),
                                  len(pairs), float(s), ptr(out), stream_ptr()), "pb_pair_products")
    _count((len(pairs) + 255) // 256)
    return out


def shell_rows(grid, F, Q, modes, row_key, out_row, scale, out, ws):
    """Rows of out (n, n_cols) FP64 for one shell; row_key/out_row host int lists (<= 32 each)."""
    lib = load()
    rk = np.ascontiguousarray(row_key, dtype=np.int32)
    orow = np.ascontiguousarray(out_row, dtype=np.int32)
    n_modes = modes.numel()
    nbytes = ctypes.c_size_t()
    check(lib.pb_shell_rows_workspace_size(n_modes, len(rk), Q.shape[0], ctypes.byref(nbytes)),
          "pb_shell_rows_workspace_size")
    buf = ws.get(nbytes.value, "shellrows")
    check(lib.pb_shell_rows(ctypes.byref(grid), precision_of(F.dtype), ptr(F), F.shape[0], ptr(Q), Q.shape[0],
                            ptr(modes), n_modes, hptr(rk), hptr(orow), len(rk), float(scale), ptr(out),
                            out.shape[-1], ptr(buf), buf.numel(), stream_ptr()), "pb_shell_rows")
    _count(2)


_tc = None


def tc_built():
    """True when libpb_b200 carries the tcgen05 triplet contraction."""
    global _tc
    if _tc is None:
        nbytes = ctypes.c_size_t()
        counts = np.ones(4, dtype=np.int32)
        st = load().pb_triplet_workspace_size(PB_F32, PB_TRIPLET_TC, 1 << 20, hptr(counts), 1, ctypes.byref(nbytes))
        _tc = (st == 0)
    return _tc


def binned_filter(grid, src, out, edges, ells, coef, w=None, wpow=0, scale=1.0):
    """out(k) = scale * src(k) * w^wpow * sum_e coef[e, bin(k)] L_ells[e](mu); coef device FP64 (n_ell, nk)."""
    edges = np.ascontiguousarray(edges, dtype=np.float64)
    ells = np.ascontiguousarray(np.asarray(ells, dtype=np.int32).reshape(-1))
    coef = coef.to(torch.float64).contiguous()
    check(load().pb_binned_filter(ctypes.byref(grid), precision_of(src.dtype), ptr(src), ptr(out), hptr(edges),
                                  len(edges) - 1, hptr(ells), len(ells), ptr(coef), ptr(w), int(wpow), float(scale),
                                  stream_ptr()), "pb_binned_filter")
    _count(1)
    return out


def shell_synth(grid, precision, src, out, maps, out_n, ws, w=None, src_stride=None):
    """Real maps out[m] = unnormalised c2r on grid out_n of the filter `maps` (entries
    (src_idx, lo, hi, l1, l2, scale, wpow) as spectral_filter) in one pruned pass per chunk
    of 64 maps.  out: a (n_maps, *out_n) tensor, or a TiledMaps set of f32 maps (one pass:
    at most 64 maps).  Raises NotImplementedError when the band limits do not allow it."""
    lib = load()
    if isinstance(out, TiledMaps):
        return _shell_synth_tiled(lib, grid, precision, src, out, maps, out_n, ws, w, src_stride)
    on = np.ascontiguousarray(out_n, dtype=np.int32)
    stride = src_stride if src_stride is not None else (src[0].numel() if src is not None and src.dim() == 4 else 0)
    c0 = 0
    while c0 < len(maps):
        # at most 64 maps, and fewer while the transform workspace would exceed SYNTH_WS_BYTES
        nc = min(SYNTH_MAX_MAPS, len(maps) - c0)
        while True:
            hi_c = np.ascontiguousarray(np.asarray(maps[c0:c0 + nc], dtype=np.float64)[:, 2])
            nbytes = ctypes.c_size_t()
            check(lib.pb_shell_synth_workspace_size(ctypes.byref(grid), hptr(on), precision, nc, hptr(hi_c),
                                                    ctypes.byref(nbytes)), "pb_shell_synth_workspace_size")
            if nbytes.value <= SYNTH_WS_BYTES or nc == 1:
                break
            nc = (nc + 1) // 2
        chunk = maps[c0:c0 + nc]
        arr = np.asarray(chunk, dtype=np.float64)
        si = np.ascontiguousarray(arr[:, 0].astype(np.int32))
        lo = np.ascontiguousarray(arr[:, 1])
        hi = np.ascontiguousarray(arr[:, 2])
        l1 = np.ascontiguousarray(arr[:, 3].astype(np.int32))
        l2 = np.ascontiguousarray(arr[:, 4].astype(np.int32))
        sc = np.ascontiguousarray(arr[:, 5])
        wp = np.ascontiguousarray(arr[:, 6].astype(np.int32))
        nbytes = ctypes.c_size_t()
        check(lib.pb_shell_synth_workspace_size(ctypes.byref(grid), hptr(on), precision, len(chunk), hptr(hi),
                                                ctypes.byref(nbytes)), "pb_shell_synth_workspace_size")
        buf = ws.get(nbytes.value, "synth")
        check(lib.pb_shell_synth(ctypes.byref(grid), hptr(on), precision, ptr(src), stride, len(chunk), hptr(si),
                                 hptr(lo), hptr(hi), hptr(l1), hptr(l2), hptr(sc), hptr(wp), ptr(w),
                                 ptr(out[c0:c0 + len(chunk)]), ptr(buf), buf.numel(), stream_ptr()), "pb_shell_synth")
        _count(3)
        c0 += nc
    return out


def _shell_synth_tiled(lib, grid, precision, src, out, maps, out_n, ws, w, src_stride):
    if precision not in (PB_F32, PB_F32_SRC_F64):
        raise ValueError("shell_synth: a tiled set holds f32 maps")
    if len(maps) != out.n_maps or tuple(int(n) for n in out_n) != out.shape:
        raise ValueError("shell_synth: the tiled set holds %d maps on %s" % (out.n_maps, out.shape))
    if len(maps) > SYNTH_MAX_MAPS:
        raise NotImplementedError("shell_synth: a tiled set is synthesised in one pass of at most 64 maps")
    on = np.ascontiguousarray(out_n, dtype=np.int32)
    stride = src_stride if src_stride is not None else (src[0].numel() if src is not None and src.dim() == 4 else 0)
    arr = np.asarray(maps, dtype=np.float64)
    si = np.ascontiguousarray(arr[:, 0].astype(np.int32))
    lo, hi, sc = (np.ascontiguousarray(arr[:, k]) for k in (1, 2, 5))
    l1, l2, wp = (np.ascontiguousarray(arr[:, k].astype(np.int32)) for k in (3, 4, 6))
    nbytes = ctypes.c_size_t()
    check(lib.pb_shell_synth_workspace_size(ctypes.byref(grid), hptr(on), precision, len(maps), hptr(hi),
                                            ctypes.byref(nbytes)), "pb_shell_synth_workspace_size")
    if nbytes.value > SYNTH_WS_BYTES:
        raise NotImplementedError("shell_synth: a tiled set's transform workspace exceeds SYNTH_WS_BYTES")
    buf = ws.get(nbytes.value, "synth")
    check(lib.pb_shell_synth_tiled(ctypes.byref(grid), hptr(on), precision, ptr(src), stride, len(maps),
                                   out.n_factor, hptr(si),
                                   hptr(lo), hptr(hi), hptr(l1), hptr(l2), hptr(sc), hptr(wp), ptr(w),
                                   ptr(out.data), ptr(buf), buf.numel(), stream_ptr()), "pb_shell_synth_tiled")
    _count(3)
    return out


class BilinearPlan:
    """Device table of pb_bilinear_plan for host terms (o, i, j, c)."""

    def __init__(self, n_g, n_out, o, i, j, c, device):
        lib = load()
        o = np.ascontiguousarray(o, dtype=np.int32)
        i = np.ascontiguousarray(i, dtype=np.int32)
        j = np.ascontiguousarray(j, dtype=np.int32)
        c = np.ascontiguousarray(c, dtype=np.float64)
        nbytes = ctypes.c_size_t()
        n = np.zeros(1, dtype=np.int32)
        check(lib.pb_bilinear_plan(n_g, n_out, hptr(o), hptr(i), hptr(j), hptr(c), len(o), None, ctypes.byref(nbytes),
                                   hptr(n)), "pb_bilinear_plan")
        host = np.zeros(nbytes.value, dtype=np.uint8)
        check(lib.pb_bilinear_plan(n_g, n_out, hptr(o), hptr(i), hptr(j), hptr(c), len(o), hptr(host),
                                   ctypes.byref(nbytes), hptr(n)), "pb_bilinear_plan")
        self.n_g, self.n_out, self.n_table = n_g, n_out, int(n[0])
        self.table = torch.from_numpy(host).to(device)

    def maps(self, G, out=None):
        """out[o] = sum_t c_t G[i_t] G[j_t]; G (n_g, ...) real maps."""
        if G.shape[0] != self.n_g:
            raise ValueError("BilinearPlan.maps: the plan was built for %d maps" % self.n_g)
        if out is None:
            out = torch.empty((self.n_out,) + tuple(G.shape[1:]), dtype=G.dtype, device=G.device)
        check(load().pb_bilinear_maps(precision_of(G.dtype), G[0].numel(), ptr(G), self.n_g, ptr(self.table),
                                      self.n_table, self.n_out, ptr(out), stream_ptr()), "pb_bilinear_maps")
        _count(1)
        return out
