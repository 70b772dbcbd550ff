"""CPU-side checks of the C-ABI library: it loads, exports every entry point that
include/polybin3d_b200.h declares, validates arguments before touching a device, and the
host-only triplet planner covers every triplet exactly once."""
import ctypes
import os
import re

import numpy as np
import pytest

from polybin3d_b200 import _native as nat

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(REPO, "include", "polybin3d_b200.h")


def declared():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"PB_API\s+(?:int|const char \*)\s*(pb_\w+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    lib = nat.load()
    names = declared()
    assert len(names) >= 10
    for n in names:
        assert hasattr(lib, n), n
    assert set(nat.SIGNATURES) >= set(names) - set(), set(names) - set(nat.SIGNATURES)
    assert lib.pb_abi_version() == 2


def test_invalid_grid_rejected_without_device():
    lib = nat.load()
    g = nat.PBGrid()
    g.n[0], g.n[1], g.n[2] = 8, 8, 7
    for i in range(3):
        g.kf[i] = 0.1
    h = ctypes.c_void_p()
    ws = ctypes.c_size_t()
    st = lib.pb_fft_plan_create(ctypes.byref(g), 1, 1, 0, ctypes.byref(h), ctypes.byref(ws))
    assert st == -1
    assert b"Last dimension of grid must be even" in lib.pb_last_error()
    with pytest.raises(ValueError, match="Last dimension"):
        nat.check(st)


def test_zero_line_of_sight_rejected():
    """A grid that asks for a line of sight (local sightline) must give a non-zero one."""
    lib = nat.load()
    g = nat.PBGrid()
    g.n[0] = g.n[1] = g.n[2] = 8
    for i in range(3):
        g.kf[i] = 0.1
    g.flags = nat.PB_GRID_LOS
    h = ctypes.c_void_p()
    ws = ctypes.c_size_t()
    st = lib.pb_fft_plan_create(ctypes.byref(g), 1, 1, 0, ctypes.byref(h), ctypes.byref(ws))
    assert st == -1 and b"line of sight must be a non-zero vector" in lib.pb_last_error()


def test_bin_reduce_argument_checks():
    lib = nat.load()
    g = nat.PBGrid()
    g.n[0] = g.n[1] = g.n[2] = 8
    for i in range(3):
        g.kf[i] = 0.1
    edges = np.array([0.1, 0.3, 0.2])
    ells = np.zeros(2, dtype=np.int32)
    st = lib.pb_bin_reduce(ctypes.byref(g), 1, 2, None, None, 1, 0, nat.hptr(edges), 2, nat.hptr(ells), 1, 1.0,
                           ctypes.c_void_p(8), 0, ctypes.c_void_p(8), 1 << 20, None)
    assert st == -1 and b"strictly increasing" in lib.pb_last_error()


def test_triplet_plan_covers_each_triplet_once():
    rng = np.random.default_rng(1)
    for n_maps, n_trip in [(10, 40), (32, 888), (48, 1500)]:
        idx = []
        seen = set()
        while len(idx) < n_trip:
            t = tuple(int(v) for v in rng.integers(0, n_maps, 3))
            if t not in seen:
                seen.add(t)
                idx.append(t)
        idx = np.asarray(idx, dtype=np.int32)
        lib = nat.load()
        nb = ctypes.c_size_t()
        counts = np.zeros(4, dtype=np.int32)
        nat.check(lib.pb_triplet_plan(n_maps, n_maps, n_maps, nat.hptr(idx), n_trip, None, ctypes.byref(nb),
                                      nat.hptr(counts)))
        host = np.zeros(nb.value, dtype=np.uint8)
        nat.check(lib.pb_triplet_plan(n_maps, n_maps, n_maps, nat.hptr(idx), n_trip, nat.hptr(host),
                                      ctypes.byref(nb), nat.hptr(counts)))
        n_items, n_pairs, n_groups = int(counts[0]), int(counts[1]), int(counts[2])
        assert counts[3] == n_trip
        rec = host[:n_items * 180].view(np.int32).reshape(n_items, -1)   # a, b[4], c[8], out[4][8]
        got = {}
        for r in rec:
            a, bs, cs, out = r[0], r[1:5], r[5:13], r[13:45].reshape(4, 8)
            for i in range(4):
                for j in range(8):
                    if out[i, j] >= 0:
                        assert out[i, j] not in got
                        got[out[i, j]] = (a, bs[i], cs[j])
        assert len(got) == n_trip
        for t, v in got.items():
            assert tuple(idx[t]) == tuple(int(x) for x in v)
        # tensor-core section: pairs sorted, groups cover every pair row, tmap consistent
        a16 = lambda x: (x + 15) // 16 * 16
        off_p = a16(n_items * 180)
        off_g = a16(off_p + n_pairs * 8)
        off_t = a16(off_g + n_groups * 16)
        pairs = host[off_p:off_p + n_pairs * 8].view(np.int32).reshape(-1, 2)
        assert [tuple(p) for p in pairs] == sorted({(int(a), int(b)) for a, b, _ in idx})
        groups = host[off_g:off_g + n_groups * 16].view(np.int32).reshape(-1, 4)
        covered = []
        for a, row0, cnt, _ in groups:
            assert 1 <= cnt <= 4
            for r in range(row0, row0 + cnt):
                assert pairs[r][0] == a
                covered.append(r)
        assert covered == list(range(n_pairs))
        tmap = host[off_t:off_t + n_trip * 8].view(np.int32).reshape(-1, 2)
        for t in range(n_trip):
            assert tuple(pairs[tmap[t, 0]]) == (idx[t, 0], idx[t, 1]) and tmap[t, 1] == idx[t, 2]


def test_triplet_plan_rejects_out_of_range():
    lib = nat.load()
    idx = np.array([[0, 1, 5]], dtype=np.int32)
    nb = ctypes.c_size_t()
    counts = np.zeros(4, dtype=np.int32)
    st = lib.pb_triplet_plan(4, 4, 4, nat.hptr(idx), 1, None, ctypes.byref(nb), nat.hptr(counts))
    assert st == -1 and b"out of range" in lib.pb_last_error()


def test_triplet_plan_rejects_duplicates():
    """A repeated (a, b, c) row would leave one output unwritten: refused."""
    lib = nat.load()
    idx = np.array([[0, 1, 2], [1, 1, 2], [0, 1, 2]], dtype=np.int32)
    nb = ctypes.c_size_t()
    counts = np.zeros(4, dtype=np.int32)
    st = lib.pb_triplet_plan(4, 4, 4, nat.hptr(idx), 3, None, ctypes.byref(nb), nat.hptr(counts))
    assert st == -1 and b"duplicate triplet at row 2" in lib.pb_last_error()


def test_bilinear_plan_host_logic():
    """pb_bilinear_plan: i <= j canonical order, duplicates merged, empty outputs get a zero
    term, out-of-range indices refused (host only)."""
    import ctypes
    from polybin3d_b200 import _native as nat
    lib = nat.load()
    o = np.array([1, 1, 0, 1], dtype=np.int32)
    i = np.array([3, 0, 2, 3], dtype=np.int32)
    j = np.array([0, 3, 2, 0], dtype=np.int32)
    c = np.array([1.0, 2.0, 0.5, 4.0])
    nb = ctypes.c_size_t()
    n = np.zeros(1, dtype=np.int32)
    assert lib.pb_bilinear_plan(4, 3, nat.hptr(o), nat.hptr(i), nat.hptr(j), nat.hptr(c), 4, None,
                                ctypes.byref(nb), nat.hptr(n)) == 0
    buf = np.zeros(nb.value, dtype=np.uint8)
    assert lib.pb_bilinear_plan(4, 3, nat.hptr(o), nat.hptr(i), nat.hptr(j), nat.hptr(c), 4, nat.hptr(buf),
                                ctypes.byref(nb), nat.hptr(n)) == 0
    k = int(n[0])
    head = ((3 + 1) * 4 + 15) // 16 * 16
    offs = buf[:16].view(np.int32)[:4]
    assert list(offs) == [0, 1, 2, 2]                     # output 2 has no term
    rec = buf[head:].reshape(k, 16)
    code = rec[:, :4].copy().view(np.uint32)[:, 0]
    coef = rec[:, 8:].copy().view(np.float64)[:, 0]
    rows = [(int((x >> 8) & 0xFF), int(x & 0xFF), float(e)) for x, e in zip(code, coef)]
    assert rows == [(2, 2, 0.5), (0, 3, 7.0)]
    assert [int((x >> 16) & 1) for x in code] == [1, 1]
    bad = np.array([5], dtype=np.int32)
    assert lib.pb_bilinear_plan(4, 3, nat.hptr(o[:1]), nat.hptr(bad), nat.hptr(j[:1]), nat.hptr(c[:1]), 1, None,
                                ctypes.byref(nb), nat.hptr(n)) != 0


def test_tuning_settings_round_trip_and_checks():
    """pb_set_tuning / pb_get_tuning need no device: settings are per host thread, zero means
    the default, out-of-range values are refused and NULL restores every default."""
    cfg = {"tc_tile": 32, "tc_stages": 3, "tc_chain": 2048, "red_method": 1, "red_warps": 2, "red_waves": 4,
           "tc_wait": 2, "tc_dsets": 1}
    nat.set_tuning(cfg)
    try:
        assert nat.get_tuning() == cfg
        for bad in ({"tc_tile": 48}, {"tc_stages": 9}, {"tc_chain": 1000}, {"red_method": 3}, {"red_warps": 9},
                    {"red_waves": -1}, {"tc_wait": 3}, {"tc_dsets": 3}):
            with pytest.raises(ValueError):
                nat.set_tuning(bad)
        assert nat.get_tuning()["tc_tile"] == 32  # a refused setting leaves the previous one
    finally:
        nat.set_tuning(None)
    assert all(v == 0 for v in nat.get_tuning().values())


def test_tiled_map_layout_host_side():
    """Tiled map sets: the size covers whole 128-voxel tiles of [factor slabs][C operand], the
    byte offsets of the FP32 factor values and of the bf16 hi / lo parts (as the header states
    them) never collide and stay inside that size, a map's 32 (factor) consecutive voxels fill
    one 128-byte row and 16 (operand) one 32-byte sector, and the converters refuse bad
    arguments without a device."""
    lib = nat.load()
    for n_maps, n_factor, n_vox in ((1, 1, 1), (5, 3, 1000), (32, 16, 192 ** 3 // 64), (33, 33, 50_003)):
        F, P = (n_factor + 7) // 8 * 8, (n_maps + 15) // 16 * 16
        size = (n_vox + 127) // 128 * 512 * (F + P)
        assert nat.tiled_maps_bytes(n_maps, n_factor, n_vox) == size
        fo = nat.tiled_factor_offsets(n_maps, n_factor, n_vox)
        co = nat.tiled_c_offsets(n_maps, n_factor, n_vox)
        assert fo.min() >= 0 and fo.max() + 4 <= size and co.min() >= 0 and co.max() + 2 <= size
        spans = np.concatenate([(fo // 4).reshape(-1) * 2, (fo // 4).reshape(-1) * 2 + 1, (co // 2).reshape(-1)])
        assert len(np.unique(spans)) == spans.size  # in 2-byte units: no overlaps
        v = np.arange(n_vox)
        for m in (0, n_factor - 1):
            assert np.all(fo[m] // 128 == fo[m][v - v % 32] // 128)
        for m in (0, n_maps - 1):
            assert np.all(co[0, m] // 32 == co[0, m][v - v % 16] // 32)
    nb = ctypes.c_size_t()
    assert lib.pb_tiled_maps_bytes(0, 1, 10, ctypes.byref(nb)) != 0
    assert lib.pb_tiled_maps_bytes(4, 5, 10, ctypes.byref(nb)) != 0
    assert lib.pb_tiled_maps_bytes(4, 0, 10, ctypes.byref(nb)) != 0
    assert lib.pb_tile_maps(None, 4, 2, 100, None, None) != 0
    counts = np.ones(4, dtype=np.int32)
    out = np.zeros(1)
    # NULL maps and a factor count outside [1, n_maps] are refused before any device work
    assert lib.pb_triplet_contract_tiled(nat.PB_TRIPLET_TC, None, 4, 2, 100, nat.hptr(counts), nat.hptr(counts), 1.0,
                                         nat.hptr(out), None, 0, None) != 0


def test_binding_constants_match_header():
    """Every PB_* constant the Python binding defines has the header's value, and the new
    argument values are refused where they do not apply (no device work)."""
    src = open(HEADER).read()
    defs = {m.group(1): int(m.group(2)) for m in re.finditer(r"^#define (PB_[A-Z0-9_]+) +\(?(-?\d+)\)?", src, re.M)}
    names = [k for k in dir(nat) if k.startswith("PB_")]
    assert names
    for k in names:
        assert k in defs, k
        assert getattr(nat, k) == defs[k], k
    lib = nat.load()
    # WIDEN reads FP32 only; NULL pointers are refused before any launch
    assert lib.pb_elementwise(nat.PB_F64, nat.PB_EW_WIDEN, 4, None, None, 0, None, None, 0.0, None, None) != 0
    assert lib.pb_elementwise(nat.PB_F32, nat.PB_EW_WIDEN, 4, None, None, 0, None, None, 0.0, None, None) != 0
    assert lib.pb_elementwise(nat.PB_F32, 7, 4, None, None, 0, None, None, 0.0, None, None) != 0
