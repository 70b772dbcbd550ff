"""Tiled map sets (the tensor-core contraction's staging layout in device memory: FP32 pair
factor maps and the bf16 hi/lo C operand per 128-voxel tile): conversion, the pruned
synthesis writing the layout directly (identical values to its plain output), and the
tensor-core contraction from a tiled set (one contiguous bulk copy per tile, the MMA reading
the operand from the staged tile) against FP64 sums and against the same contraction from
plain maps; the bispectrum estimator through the tiled path against the plain path."""
import contextlib
import ctypes
import io

import numpy as np
import pytest
import torch

from polybin3d_b200 import _native as nat

pytestmark = pytest.mark.gpu

tc = pytest.mark.skipif(not (torch.cuda.is_available() and torch.cuda.get_device_capability()[0] == 10
                             and nat.tc_built()), reason="tensor-core contraction needs sm_100")


def bk_like_triplets(nk=16, lmax=2):
    kc = np.arange(nk) + 0.5
    rows = []
    for l in range(0, lmax + 1, 2):
        for b1 in range(nk):
            for b2 in range(b1, nk):
                for b3 in range(b2, nk):
                    if abs(kc[b1] - kc[b2]) <= kc[b3] <= kc[b1] + kc[b2]:
                        rows.append((b1, b2, (l // 2) * nk + b3))
    return np.asarray(rows, dtype=np.int32)


def reference(G, idx):
    G = G.double()
    out = torch.empty(len(idx), dtype=torch.float64, device=G.device)
    for t0 in range(0, len(idx), 64):
        sl = idx[t0:t0 + 64]
        out[t0:t0 + len(sl)] = (G[sl[:, 0]] * G[sl[:, 1]] * G[sl[:, 2]]).sum(dim=1)
    return out


def split(G):
    hi = G.to(torch.bfloat16)
    return hi, (G - hi.float()).to(torch.bfloat16)


def covered(T):
    """Bool mask over T.data of the bytes the layout assigns to the set's voxels."""
    hit = torch.zeros(T.data.numel(), dtype=torch.bool, device=T.data.device)
    fo = torch.as_tensor(nat.tiled_factor_offsets(T.n_maps, T.n_factor, T.n_vox), device=hit.device).reshape(-1)
    co = torch.as_tensor(nat.tiled_c_offsets(T.n_maps, T.n_factor, T.n_vox), device=hit.device).reshape(-1)
    for o, w in ((fo, 4), (co, 2)):
        for k in range(w):
            hit[o + k] = True
    return hit


@pytest.mark.parametrize("n_maps,n_factor,n_vox", [(5, 3, 50_003), (32, 16, 64 ** 3), (33, 33, 1000)])
def test_tile_maps_round_trip(n_maps, n_factor, n_vox):
    torch.manual_seed(0)
    G = torch.randn(n_maps, n_vox, device="cuda")
    T = nat.TiledMaps.from_maps(G, n_factor)
    assert torch.equal(T.factor_maps(), G[:n_factor])
    hi, lo = T.split_parts()
    rh, rl = split(G)
    assert torch.equal(hi, rh) and torch.equal(lo, rl)
    # padding rows and the voxels past n_vox are zero
    assert torch.count_nonzero(T.data[~covered(T)]) == 0


@tc
@pytest.mark.parametrize("n_vox", [64 ** 3, 50_003, 128])
@pytest.mark.parametrize("cfg", [{}, {"tc_stages": 2}, {"tc_wait": 2}, {"tc_dsets": 1}])
def test_contract_tiled_matches_fp64(n_vox, cfg):
    """32 maps (16 pair factors), 136 pairs (128 in tensor memory + 8 side pairs), 888 triplets."""
    torch.manual_seed(1)
    idx = bk_like_triplets()
    G = torch.randn(32, n_vox, device="cuda")
    ref = reference(G, torch.as_tensor(idx, device="cuda").long()).cpu().numpy()
    ws = nat.Workspace(torch.device("cuda"))
    plan = nat.TripletPlan(32, 32, 32, idx, torch.device("cuda"))
    T = nat.TiledMaps.from_maps(G, 16)
    out = torch.empty(len(idx), dtype=torch.float64, device="cuda")
    nat.set_tuning(cfg)
    try:
        for _ in range(2):
            out.fill_(0.0)
            plan.contract_tiled(T, out, ws)
            got = out.cpu().numpy()
            assert np.all(np.isfinite(got))
            assert np.max(np.abs(got - ref)) / np.max(np.abs(ref)) < 1e-5
    finally:
        nat.set_tuning(None)
    plain = torch.empty_like(out)
    plan.contract(G, G, G, plain, ws, method=nat.PB_TRIPLET_TC)
    assert np.max(np.abs(plain.cpu().numpy() - got)) / np.max(np.abs(ref)) < 1e-5


@tc
@pytest.mark.parametrize("nk", [24, 12])
def test_contract_tiled_other_shapes(nk):
    """48 maps / 300 pairs (M-tiles that do not fit two 128-voxel operand buffers: pair
    chunks) and 24 maps / 78 pairs (one partly filled M-tile, operand rows padded to 32)."""
    torch.manual_seed(2)
    idx = bk_like_triplets(nk=nk, lmax=2)
    n = 2 * nk
    G = torch.randn(n, 40 ** 3, device="cuda")
    ref = reference(G, torch.as_tensor(idx, device="cuda").long()).cpu().numpy()
    ws = nat.Workspace(torch.device("cuda"))
    plan = nat.TripletPlan(n, n, n, idx, torch.device("cuda"))
    out = torch.empty(len(idx), dtype=torch.float64, device="cuda")
    plan.contract_tiled(nat.TiledMaps.from_maps(G, nk), out, ws)
    got = out.cpu().numpy()
    assert np.max(np.abs(got - ref)) / np.max(np.abs(ref)) < 1e-5


@tc
def test_contract_tiled_rejects_pairs_outside_the_factor_maps():
    """A plan whose pair factors are not among the set's factor maps: the Python wrapper
    refuses it, and through the C ABI the kernel rejects it before any work (NaN outputs)."""
    torch.manual_seed(3)
    G = torch.randn(8, 4096, device="cuda")
    idx = np.asarray([(0, 1, 2), (1, 5, 3)], dtype=np.int32)
    plan = nat.TripletPlan(8, 8, 8, idx, torch.device("cuda"))
    T = nat.TiledMaps.from_maps(G, 4)
    ws = nat.Workspace(torch.device("cuda"))
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    with pytest.raises(ValueError):
        plan.contract_tiled(T, out, ws)
    buf = ws.get(plan.workspace_bytes(nat.PB_F32, nat.PB_TRIPLET_TC, T.n_vox), "triplet")
    st = nat.load().pb_triplet_contract_tiled(nat.PB_TRIPLET_TC, nat.ptr(T.data), 8, 4, T.n_vox, nat.ptr(plan.table),
                                              nat.hptr(plan.counts), 1.0, nat.ptr(out), nat.ptr(buf), buf.numel(),
                                              nat.stream_ptr())
    assert st == 0
    assert torch.isnan(out).all()


def quiet(fn, *a, **k):
    with contextlib.redirect_stdout(io.StringIO()):
        return fn(*a, **k)


@pytest.mark.parametrize("N", [40, 64])
def test_shell_synth_tiled_equals_plain(N):
    """The g-maps written as a tiled set hold exactly the values (FP32 factors, bf16 parts) of
    the plain synthesis (the 40^3 grid's 30^3 map grid ends in a partly filled tile, whose
    padding reads as zeros)."""
    import polybin3d_b200 as pb
    from polybin3d_b200 import synthetic
    L = 1000.0
    b = quiet(pb.PolyBin3D, [L] * 3, [N] * 3, pixel_window="tsc", backend="cuda", precision="mixed")
    edges = np.linspace(2 * np.pi / L, 0.3 * np.pi * N / L, 9)
    bs = quiet(pb.BSpec, b, edges, lmax=2)
    x = b.as_device(synthetic.lognormal(N, L, seed=3))
    xk = bs._data_spectrum(x)
    w = bs._data_weight(torch.float32)
    G = bs._g_maps(xk, w, 1.0).reshape(2 * bs.Nk_squeeze, -1)
    T = bs._g_maps_tiled(xk, w, 1.0)
    assert T is not None and T.n_vox == G.shape[1] and T.n_factor == bs.Nk_squeeze
    assert torch.equal(T.factor_maps().reshape(T.n_factor, -1), G[:T.n_factor])
    hi, lo = T.split_parts()
    rh, rl = split(G)
    assert torch.equal(hi.reshape(T.n_maps, -1), rh) and torch.equal(lo.reshape(T.n_maps, -1), rl)
    if T.n_vox % 128:
        nv = (T.n_vox + 127) // 128 * 128
        fo = nat.tiled_factor_offsets(T.n_maps, T.n_factor, nv)[:, T.n_vox:].reshape(-1)
        co = nat.tiled_c_offsets(T.n_maps, T.n_factor, nv)[:, :, T.n_vox:].reshape(-1)
        pad = torch.as_tensor(np.concatenate([fo, fo + 1, fo + 2, fo + 3, co, co + 1]), device=T.data.device)
        assert torch.count_nonzero(T.data[pad]) == 0


@tc
def test_bk_routes_agree():
    """The bispectrum's cubic sums through the tiled set and through plain maps (mixed
    precision, tensor cores) on one field: the same sums up to FP32 accumulation order within
    tiles; Bk_numerator_ideal returns the route the autotuner picked."""
    import polybin3d_b200 as pb
    from polybin3d_b200 import synthetic
    N, L = 64, 1000.0
    b = quiet(pb.PolyBin3D, [L] * 3, [N] * 3, pixel_window="tsc", backend="cuda", precision="mixed")
    bs = quiet(pb.BSpec, b, np.linspace(2 * np.pi / L, 0.15, 9), lmax=2, contraction="tc")
    bs.sym_factor = np.ones(bs.N_bins)
    field = synthetic.lognormal(N, L, seed=4)
    assert bs._tiled_ok(torch.float32)
    x = b.as_device(field)
    f32 = torch.float32
    xk = bs._data_spectrum(x, keep64=True)  # as Bk_ideal: FP32 maps from the FP64 transform
    w = bs._data_weight(f32)
    scale = 1.0 / bs.cube_mask_mean ** (1. / 3.)
    tiled = bs._b3_tiled(xk, w, scale, f32).cpu().numpy()
    plain = bs._b3_plain(xk, w, scale, f32).cpu().numpy()
    nb = len(plain) // 2
    for j in range(2):
        a, r = tiled[j * nb:(j + 1) * nb], plain[j * nb:(j + 1) * nb]
        assert np.max(np.abs(a - r)) / np.max(np.abs(r)) < 1e-6
    num = quiet(bs.Bk_numerator_ideal, field)
    norm = b.volume / float(b.gridsize.prod())
    ref = tiled if bs._b3_route(xk, w, scale, f32) == "tiled" else plain
    assert np.max(np.abs(num / norm - ref)) / np.max(np.abs(ref)) < 1e-12
