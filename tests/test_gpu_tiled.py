"""Tiled map sets (the tensor-core contraction's staging layout in device memory):
conversion round trip, the pruned synthesis writing the layout directly (identical values
to its plain output), and the tensor-core contraction from a tiled set (one contiguous bulk
copy per tile) against FP64 sums and against the same contraction from plain maps; the
bispectrum estimator through the tiled path against the plain path."""
import contextlib
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


@pytest.mark.parametrize("n_maps,n_vox", [(5, 50_003), (32, 64 ** 3), (33, 1000)])
def test_tile_maps_round_trip(n_maps, n_vox):
    torch.manual_seed(0)
    G = torch.randn(n_maps, n_vox, device="cuda")
    T = nat.TiledMaps.from_maps(G)
    assert torch.equal(T.to_maps(), G)
    # everything the index does not reach (padding rows, voxels past n_vox) is zero
    hit = torch.zeros(T.data.numel(), dtype=torch.bool, device="cuda")
    hit[torch.as_tensor(nat.tiled_index(n_maps, n_vox), device="cuda").reshape(-1)] = True
    assert torch.count_nonzero(T.data[~hit]) == 0


@tc
@pytest.mark.parametrize("n_vox", [64 ** 3, 50_003, 128])
@pytest.mark.parametrize("cfg", [{}, {"tc_tile": 64}, {"tc_tile": 32}, {"tc_stages": 2}])
def test_contract_tiled_matches_fp64(n_vox, cfg):
    """32 maps, 136 pairs (128 in tensor memory + 8 side pairs), 888 triplets."""
    torch.manual_seed(1)
    idx = bk_like_triplets()
    G = torch.randn(32, n_vox, device="cuda")
    ref = reference(G, torch.as_tensor(idx, device="cuda").long()).cpu().numpy()
    ws = nat.Workspace(torch.device("cuda"))
    plan = nat.TripletPlan(32, 32, 32, idx, torch.device("cuda"))
    T = nat.TiledMaps.from_maps(G)
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
    """48 maps / 300 pairs (pair M-tiles that do not fit 128-voxel operand buffers: smaller
    tiles) and 24 maps / 78 pairs (one partly filled M-tile)."""
    torch.manual_seed(2)
    idx = bk_like_triplets(nk=nk, lmax=2)
    n = 2 * nk
    G = torch.randn(n, 40 ** 3, device="cuda")
    ref = reference(G, torch.as_tensor(idx, device="cuda").long()).cpu().numpy()
    ws = nat.Workspace(torch.device("cuda"))
    plan = nat.TripletPlan(n, n, n, idx, torch.device("cuda"))
    out = torch.empty(len(idx), dtype=torch.float64, device="cuda")
    plan.contract_tiled(nat.TiledMaps.from_maps(G), out, ws)
    got = out.cpu().numpy()
    assert np.max(np.abs(got - ref)) / np.max(np.abs(ref)) < 1e-5


@tc
def test_contract_tiled_refuses_a_foreign_plan():
    G = torch.randn(8, 4096, device="cuda")
    idx = np.asarray([(0, 1, 2), (1, 2, 3)], dtype=np.int32)
    plan = nat.TripletPlan(8, 8, 4, idx, torch.device("cuda"))
    with pytest.raises(ValueError):
        plan.contract_tiled(nat.TiledMaps.from_maps(G), torch.empty(2, dtype=torch.float64, device="cuda"),
                            nat.Workspace(torch.device("cuda")))


def quiet(fn, *a, **k):
    with contextlib.redirect_stdout(io.StringIO()):
        return fn(*a, **k)


@pytest.mark.parametrize("N", [40, 64])
def test_shell_synth_tiled_equals_plain(N):
    """The g-maps written as a tiled set hold exactly the values of the plain synthesis (the
    40^3 grid's 30^3 map grid ends in a partly filled 128-voxel tile)."""
    import polybin3d_b200 as pb
    from polybin3d_b200 import synthetic
    L = 1000.0
    b = quiet(pb.PolyBin3D, [L] * 3, [N] * 3, pixel_window="tsc", backend="cuda", precision="mixed")
    edges = np.linspace(2 * np.pi / L, 0.3 * np.pi * N / L, 9)
    bs = quiet(pb.BSpec, b, edges, lmax=2)
    x = b.as_device(synthetic.lognormal(N, L, seed=3))
    xk = bs._data_spectrum(x)
    w = bs._data_weight(torch.float32)
    G = bs._g_maps(xk, w, 1.0)
    T = bs._g_maps_tiled(xk, w, 1.0)
    assert T is not None and T.shape == tuple(G.shape[1:])
    assert torch.equal(T.to_maps(), G)
    if T.n_vox % 128:
        hit = torch.zeros(T.data.numel(), dtype=torch.bool, device=T.data.device)
        hit[torch.as_tensor(nat.tiled_index(T.n_maps, T.n_vox), device=hit.device).reshape(-1)] = True
        tail = torch.arange(T.data.numel(), device=hit.device) >= (T.data.numel() - 4 * 32 * ((T.n_maps + 7) // 8 * 8))
        assert torch.count_nonzero(T.data[~hit & tail]) == 0


@tc
def test_bk_ideal_tiled_path_matches_plain_path():
    """Bk_ideal (mixed precision, tensor cores) through the tiled set and through plain maps:
    the same sums up to FP32 accumulation order within tiles."""
    import polybin3d_b200 as pb
    from polybin3d_b200 import synthetic
    N, L = 64, 1000.0
    b = quiet(pb.PolyBin3D, [L] * 3, [N] * 3, pixel_window="tsc", backend="cuda", precision="mixed")
    bs = quiet(pb.BSpec, b, np.linspace(2 * np.pi / L, 0.15, 9), lmax=2, contraction="tc")
    bs.sym_factor = np.ones(bs.N_bins)
    x = synthetic.lognormal(N, L, seed=4)
    assert bs._tiled_ok(torch.float32)
    tiled = quiet(bs.Bk_numerator_ideal, x)
    assert getattr(bs, "_tiled", True)
    bs._tiled = False
    plain = quiet(bs.Bk_numerator_ideal, x)
    nb = len(plain) // 2
    for j in range(2):
        a, r = tiled[j * nb:(j + 1) * nb], plain[j * nb:(j + 1) * nb]
        assert np.max(np.abs(a - r)) / np.max(np.abs(r)) < 1e-6
