"""pb_bin_reduce_noalloc against pb_bin_reduce, through the C ABI.

The no-allocation entry point serves callers that cannot give the library device
scratch memory (a binding that only forwards the input/output pointers it received, or a
process whose GPU memory is held by another framework's pool).  Its partial sums live in a
fixed device array inside libpb_b200.so, so it must give the same answers as the
workspace-taking entry point, on consecutive calls that reuse that array, and must refuse
reductions too large for it.  This file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest
import torch

from polybin3d_b200 import _native as nat

pytestmark = pytest.mark.gpu


def _grid(n, L):
    g = nat.PBGrid()
    for i in range(3):
        g.n[i] = n
        g.kf[i] = 2 * np.pi / L
    g.flags = 0
    return g


def _reference_reduce(lib, g, prec, mode, a, b, n_rows, edges, ells):
    nk, n_ell = len(edges) - 1, len(ells) // 2
    nbytes = ctypes.c_size_t()
    nat.check(lib.pb_bin_reduce_workspace_size(ctypes.byref(g), n_rows, nk, n_ell, ctypes.byref(nbytes)))
    ws = torch.empty(nbytes.value, dtype=torch.uint8, device="cuda")
    out = torch.empty(n_rows * n_ell * nk, dtype=torch.float64, device="cuda")
    nat.check(lib.pb_bin_reduce(ctypes.byref(g), prec, mode, nat.ptr(a), nat.ptr(b), n_rows, 0, nat.hptr(edges), nk,
                                nat.hptr(ells), n_ell, 1.0, nat.ptr(out), 0, nat.ptr(ws), ws.numel(),
                                nat.stream_ptr()))
    return out


def _noalloc_reduce(lib, g, prec, mode, a, b, n_rows, edges, ells):
    nk, n_ell = len(edges) - 1, len(ells) // 2
    out = torch.full((n_rows * n_ell * nk,), np.nan, dtype=torch.float64, device="cuda")
    nat.check(lib.pb_bin_reduce_noalloc(ctypes.byref(g), prec, mode, nat.ptr(a), nat.ptr(b), n_rows, 0,
                                        nat.hptr(edges), nk, nat.hptr(ells), n_ell, 1.0, nat.ptr(out), 0,
                                        nat.stream_ptr()))
    return out


@pytest.mark.parametrize("prec,cdt", [(nat.PB_F64, torch.complex128), (nat.PB_F32, torch.complex64)])
def test_noalloc_matches_workspace_entry_point_twice(prec, cdt):
    lib = nat.load()
    n, L = 32, 500.0
    g = _grid(n, L)
    kF = 2 * np.pi / L
    edges = np.ascontiguousarray(np.linspace(kF, 0.18, 9))
    ells = np.ascontiguousarray(np.array([0, 0, 2, 0, 4, 0], dtype=np.int32))
    gen = torch.Generator(device="cuda").manual_seed(7)
    shape = (n, n, n // 2 + 1)
    # call 1: |a|^2 of one spectrum; call 2: Re(a conj b_r) for 5 rows (different slot use)
    a = torch.randn(shape, dtype=cdt, device="cuda", generator=gen)
    ref1 = _reference_reduce(lib, g, prec, nat.PB_RED_ABS2, a, None, 1, edges, ells)
    got1 = _noalloc_reduce(lib, g, prec, nat.PB_RED_ABS2, a, None, 1, edges, ells)
    b = torch.randn((5,) + shape, dtype=cdt, device="cuda", generator=gen)
    ref2 = _reference_reduce(lib, g, prec, nat.PB_RED_CROSS, a, b, 5, edges, ells)
    got2 = _noalloc_reduce(lib, g, prec, nat.PB_RED_CROSS, a, b, 5, edges, ells)
    torch.cuda.synchronize()
    for ref, got in ((ref1, got1), (ref2, got2)):
        r, o = ref.cpu().numpy(), got.cpu().numpy()
        assert np.all(np.isfinite(o))
        assert np.max(np.abs(o - r)) <= 1e-10 * np.max(np.abs(r))


def test_noalloc_at_the_scratch_limit_and_mode_counts():
    """1000 rows x 64 bins x 4 multipoles = 256000 doubles per block: only one block per row
    fits the fixed array, so the entry point runs the reduction on a one-block grid; it must
    still equal the workspace entry point, and so must the mode counts (REAL2, no input)."""
    lib = nat.load()
    n, L = 32, 500.0
    g = _grid(n, L)
    kF = 2 * np.pi / L
    edges = np.ascontiguousarray(np.linspace(kF, 0.35, 65))
    ells = np.ascontiguousarray(np.array([0, 0, 2, 0, 4, 0, 2, 2], dtype=np.int32))
    gen = torch.Generator(device="cuda").manual_seed(11)
    shape = (n, n, n // 2 + 1)
    a = torch.randn(shape, dtype=torch.complex128, device="cuda", generator=gen)
    b = torch.randn((1000,) + shape, dtype=torch.complex128, device="cuda", generator=gen)
    for _ in range(2):
        ref = _reference_reduce(lib, g, nat.PB_F64, nat.PB_RED_CROSS, a, b, 1000, edges, ells)
        got = _noalloc_reduce(lib, g, nat.PB_F64, nat.PB_RED_CROSS, a, b, 1000, edges, ells)
        r, o = ref.cpu().numpy(), got.cpu().numpy()
        assert np.all(np.isfinite(o))
        assert np.max(np.abs(o - r)) <= 1e-10 * np.max(np.abs(r))
    one = np.ascontiguousarray(np.array([0, 0], dtype=np.int32))
    ref = _reference_reduce(lib, g, nat.PB_F64, nat.PB_RED_REAL2, None, None, 1, edges, one).cpu().numpy()
    got = _noalloc_reduce(lib, g, nat.PB_F64, nat.PB_RED_REAL2, None, None, 1, edges, one).cpu().numpy()
    assert np.array_equal(got, ref)


def test_noalloc_rejects_oversized_reduction():
    lib = nat.load()
    g = _grid(16, 300.0)
    edges = np.ascontiguousarray(np.linspace(0.03, 0.15, 65))
    ells = np.ascontiguousarray(np.zeros(18, dtype=np.int32))
    out = torch.empty(1, dtype=torch.float64, device="cuda")
    a = torch.zeros((16, 16, 9), dtype=torch.complex128, device="cuda")
    # 600 rows * 64 bins * 9 multipoles > 262144 doubles of fixed scratch
    st = lib.pb_bin_reduce_noalloc(ctypes.byref(g), nat.PB_F64, nat.PB_RED_ABS2, nat.ptr(a), None, 600, 0,
                                   nat.hptr(edges), 64, nat.hptr(ells), 9, 1.0, nat.ptr(out), 0, nat.stream_ptr())
    assert st == -1
    assert b"exceeds the fixed scratch" in lib.pb_last_error()
