"""The launch-shape autotuner (polybin3d_b200/autotune.py): on first use of a shape it times
the candidate settings, stores the winner in its cache file and launches with it; the tuned
result equals the default launch's (FP32 accumulation order for the tensor-core
contraction: 1e-5 of the largest triplet sum; FP64 reduction: 1e-12)."""
import json

import numpy as np
import pytest
import torch

from polybin3d_b200 import _native as nat

pytestmark = pytest.mark.gpu


def test_tuned_contraction_is_cached_and_matches_default(tmp_path, monkeypatch):
    from polybin3d_b200 import autotune
    from polybin3d_b200.bspec import tc_available
    if not tc_available():
        pytest.skip("tensor-core contraction not available")
    monkeypatch.setenv("PB_TUNING_CACHE", str(tmp_path / "tuning.json"))
    monkeypatch.setenv("PB_AUTOTUNE", "1")
    torch.manual_seed(0)
    dev = torch.device("cuda")
    idx = np.asarray([(i, j, k) for i in range(12) for j in range(i, 12) for k in range(j, 12)], dtype=np.int32)
    G = torch.randn(12, 96 ** 3, device=dev)
    ws = nat.Workspace(dev)
    plan = nat.TripletPlan(12, 12, 12, idx, dev)
    ref = torch.empty(len(idx), dtype=torch.float64, device=dev)
    plan.contract(G, G, G, ref, ws, method=nat.PB_TRIPLET_TC)
    out = torch.empty_like(ref)
    autotune.contract(plan, G, G, G, out, ws, nat.PB_TRIPLET_TC, 1.0)
    table = json.load(open(tmp_path / "tuning.json"))
    keys = [k for k in table if k.startswith("tc|")]
    assert len(keys) == 1 and table[keys[0]] in autotune.TC_CANDIDATES
    t = autotune.tuner()
    assert len(t.timings[keys[0]]) == len(autotune.TC_CANDIDATES)
    r, o = ref.cpu().numpy(), out.cpu().numpy()
    assert np.max(np.abs(o - r)) / np.max(np.abs(r)) < 1e-5
    assert all(v == 0 for v in nat.get_tuning().values())  # defaults restored after the call
    # a second call takes the cached setting without timing again
    n_timed = len(t.timings)
    autotune.contract(plan, G, G, G, out, ws, nat.PB_TRIPLET_TC, 1.0)
    assert len(t.timings) == n_timed


def test_tuned_reduction_matches_default(tmp_path, monkeypatch):
    import contextlib
    import io
    import polybin3d_b200 as pb
    from polybin3d_b200 import autotune
    monkeypatch.setenv("PB_TUNING_CACHE", str(tmp_path / "tuning.json"))
    monkeypatch.setenv("PB_AUTOTUNE", "1")
    N, L = 48, 700.0
    with contextlib.redirect_stdout(io.StringIO()):
        b = pb.PolyBin3D([L] * 3, [N] * 3, backend="cuda")
    edges = np.linspace(2 * np.pi / L, 0.15, 13)
    ells = [(0, 0), (2, 0), (4, 0)]
    gen = torch.Generator(device="cuda").manual_seed(3)
    Q = torch.randn((40,) + b.nhalf_shape, dtype=torch.complex128, device="cuda", generator=gen)
    a = torch.randn(b.nhalf_shape, dtype=torch.complex128, device="cuda", generator=gen)
    ref = torch.zeros((40, 36), dtype=torch.float64, device="cuda")
    nat.bin_reduce(b.grid, nat.PB_F64, nat.PB_RED_CROSS, a, Q, 40, edges, ells, 0.5, ref, b.ws)
    out = torch.ones_like(ref)
    autotune.bin_reduce(b.grid, nat.PB_F64, nat.PB_RED_CROSS, a, Q, 40, edges, ells, 0.5, out, b.ws,
                        accumulate=True)
    # the candidates ran on scratch: the accumulating call added the sums exactly once
    r, o = ref.cpu().numpy(), out.cpu().numpy() - 1.0
    assert np.max(np.abs(o - r)) / np.max(np.abs(r)) < 1e-12
    table = json.load(open(tmp_path / "tuning.json"))
    assert [table[k] in autotune.RED_CANDIDATES for k in table if k.startswith("red|")] == [True]
