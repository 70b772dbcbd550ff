"""Triplet contraction through the C ABI: CUDA-core (f32, f64) and tensor-core (f32)
forms against an FP64 reference on the same random maps, including a ragged voxel count
(tail tile) and aliased / distinct map sets."""
import numpy as np
import pytest
import torch

from polybin3d_b200 import _native as nat

pytestmark = pytest.mark.gpu


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


def reference(A, B, C, idx):
    A, B, C = A.double(), B.double(), C.double()
    out = torch.empty(len(idx), dtype=torch.float64, device=A.device)
    for t0 in range(0, len(idx), 64):
        sl = idx[t0:t0 + 64]
        out[t0:t0 + len(sl)] = (A[sl[:, 0]] * B[sl[:, 1]] * C[sl[:, 2]]).sum(dim=1)
    return out


@pytest.mark.parametrize("n_vox", [64 ** 3, 50_003])
def test_methods_agree_with_fp64(n_vox):
    torch.manual_seed(0)
    idx = bk_like_triplets()
    G = torch.randn(32, n_vox, device="cuda", dtype=torch.float32)
    ref = reference(G, G, G, torch.as_tensor(idx, device="cuda").long()).cpu().numpy()
    ws = nat.Workspace(torch.device("cuda"))
    plan = nat.TripletPlan(32, 32, 32, idx, torch.device("cuda"))
    out = torch.empty(len(idx), dtype=torch.float64, device="cuda")
    scale = np.max(np.abs(ref))
    plan.contract(G, G, G, out, ws, method=nat.PB_TRIPLET_SIMT)
    assert np.max(np.abs(out.cpu().numpy() - ref)) / scale < 1e-6
    Gd = G.double()
    plan.contract(Gd, Gd, Gd, out, ws, method=nat.PB_TRIPLET_SIMT)
    assert np.max(np.abs(out.cpu().numpy() - ref)) / scale < 1e-12
    if nat.tc_built() and torch.cuda.get_device_capability()[0] == 10:
        for _ in range(2):
            plan.contract(G, G, G, out, ws, method=nat.PB_TRIPLET_TC)
            got = out.cpu().numpy()
            assert np.all(np.isfinite(got))
            assert np.max(np.abs(got - ref)) / scale < 1e-5


def test_distinct_map_sets():
    torch.manual_seed(1)
    n_vox = 40 ** 3
    A = torch.randn(8, n_vox, device="cuda")
    B = torch.randn(8, n_vox, device="cuda")
    C = torch.randn(8, n_vox, device="cuda")
    idx = np.asarray([(i, j, k) for i in range(8) for j in range(i, 8) for k in range(j, 8)], dtype=np.int32)
    ref = reference(A, B, C, torch.as_tensor(idx, device="cuda").long()).cpu().numpy()
    ws = nat.Workspace(torch.device("cuda"))
    plan = nat.TripletPlan(8, 8, 8, idx, torch.device("cuda"))
    out = torch.empty(len(idx), dtype=torch.float64, device="cuda")
    scale = np.max(np.abs(ref))
    plan.contract(A, B, C, out, ws, method=nat.PB_TRIPLET_SIMT)
    assert np.max(np.abs(out.cpu().numpy() - ref)) / scale < 1e-6
    if nat.tc_built() and torch.cuda.get_device_capability()[0] == 10:
        plan.contract(A, B, C, out, ws, method=nat.PB_TRIPLET_TC)
        assert np.max(np.abs(out.cpu().numpy() - ref)) / scale < 1e-5


def test_tc_pair_chunks():
    """300 (b1, b2) pairs x 48 maps (24 bins, lmax=2): the FP64 accumulators and pair operands
    exceed shared memory in one launch, so the tensor-core form runs the pairs in chunks."""
    torch.manual_seed(2)
    idx = bk_like_triplets(nk=24, lmax=2)
    n_vox = 48 ** 3
    G = torch.randn(48, n_vox, device="cuda", dtype=torch.float32)
    ref = reference(G, G, G, torch.as_tensor(idx, device="cuda").long()).cpu().numpy()
    ws = nat.Workspace(torch.device("cuda"))
    plan = nat.TripletPlan(48, 48, 48, idx, torch.device("cuda"))
    assert plan.n_pairs == 300
    out = torch.empty(len(idx), dtype=torch.float64, device="cuda")
    scale = np.max(np.abs(ref))
    if nat.tc_built() and torch.cuda.get_device_capability()[0] == 10:
        for _ in range(2):
            plan.contract(G, G, G, out, ws, method=nat.PB_TRIPLET_TC)
            got = out.cpu().numpy()
            assert np.all(np.isfinite(got))
            assert np.max(np.abs(got - ref)) / scale < 1e-5


@pytest.mark.parametrize("n_pairs,n_c", [(136, 32), (140, 20), (129, 64), (268, 40)])
def test_tc_side_pairs(n_pairs, n_c):
    """Pair counts a little above a multiple of 128 put the extra pairs (up to 16) in the
    shared-memory side operand instead of a 128-lane M-tile of their own; C-map counts that
    are not a multiple of 32 are padded for the side MMA (M = 64 or 128)."""
    if not (nat.tc_built() and torch.cuda.get_device_capability()[0] == 10):
        pytest.skip("tensor-core contraction not available")
    rng = np.random.default_rng(n_pairs)
    n_a = 24
    allp = [(i, j) for i in range(n_a) for j in range(i, n_a)]
    sel = rng.choice(len(allp), size=n_pairs, replace=False)
    idx = np.asarray([(allp[s][0], allp[s][1], int(rng.integers(0, n_c))) for s in sel], dtype=np.int32)
    idx = np.unique(idx, axis=0)
    torch.manual_seed(n_pairs)
    A = torch.randn(n_a, 36 ** 3, device="cuda")
    C = torch.randn(n_c, 36 ** 3, device="cuda")
    ref = reference(A, A, C, torch.as_tensor(idx, device="cuda").long()).cpu().numpy()
    ws = nat.Workspace(torch.device("cuda"))
    plan = nat.TripletPlan(n_a, n_a, n_c, idx, torch.device("cuda"))
    assert plan.n_pairs == n_pairs
    out = torch.empty(len(idx), dtype=torch.float64, device="cuda")
    scale = np.max(np.abs(ref))
    for _ in range(2):
        plan.contract(A, A, C, out, ws, method=nat.PB_TRIPLET_TC)
        got = out.cpu().numpy()
        assert np.all(np.isfinite(got))
        assert np.max(np.abs(got - ref)) / scale < 1e-5


@pytest.mark.parametrize("dtype,tol", [(torch.float64, 1e-12), (torch.float32, 1e-5)])
def test_bilinear_maps(dtype, tol):
    """pb_bilinear_maps against a torch sum of products (ragged voxel count, repeated and
    reversed pairs, an output with no terms)."""
    torch.manual_seed(3)
    n_g, n_out, n_vox = 20, 6, 33_333
    G = torch.randn(n_g, n_vox, device="cuda", dtype=torch.float64)
    rng = np.random.default_rng(3)
    n_t = 300
    o = rng.integers(0, n_out - 1, n_t)          # output n_out-1 gets no term
    i = rng.integers(0, n_g, n_t)
    j = rng.integers(0, n_g, n_t)
    c = rng.standard_normal(n_t)
    ref = torch.zeros(n_out, n_vox, dtype=torch.float64, device="cuda")
    for a, b, d, e in zip(o, i, j, c):
        ref[a] += e * G[b] * G[d]
    plan = nat.BilinearPlan(n_g, n_out, o, i, j, c, torch.device("cuda"))
    out = plan.maps(G.to(dtype)).double()
    scale = ref.abs().max()
    assert float((out - ref).abs().max() / scale) < tol
    assert float(out[n_out - 1].abs().max()) == 0.0


@pytest.mark.parametrize("tile", [128, 64, 32])
def test_tc_tile_sizes(tile):
    """The tensor-core contraction from plain maps at each tile size (128 by default; 64 and 32
    when a shape needs them or the autotuner picks them), ragged voxel count included."""
    if not (nat.tc_built() and torch.cuda.get_device_capability()[0] == 10):
        pytest.skip("tensor-core contraction needs sm_100")
    torch.manual_seed(9)
    idx = bk_like_triplets()
    G = torch.randn(32, 50_003, device="cuda")
    ref = reference(G, G, G, torch.as_tensor(idx, device="cuda").long()).cpu().numpy()
    ws = nat.Workspace(torch.device("cuda"))
    plan = nat.TripletPlan(32, 32, 32, idx, torch.device("cuda"))
    out = torch.empty(len(idx), dtype=torch.float64, device="cuda")
    nat.set_tuning({"tc_tile": tile})
    try:
        plan.contract(G, G, G, out, ws, method=nat.PB_TRIPLET_TC)
    finally:
        nat.set_tuning(None)
    assert np.max(np.abs(out.cpu().numpy() - ref)) / np.max(np.abs(ref)) < 1e-5
