"""Slice sweeps on the GPU against the reference's golden per-section counts
(data/counts-N.npy from the original solve) and against per-line compute."""
import json
import os

import numpy as np
import pytest

from tests.oracle import P

pytestmark = pytest.mark.gpu
GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "counts_30_35.npz"))


def check_golden(res):
    for s, rows in res.items():
        gold = {int(r[0]): r for r in GOLD[f"counts_{s}"]}
        for r in rows:
            assert np.array_equal(gold[int(r[0])], r), f"slice {s} section {int(r[0]):#x}"


def test_sweep_small_root_matches_golden_counts(cuda):
    """Root [[4,4],[5,4],[4,5],[4,3]] (33 stones): slices 35, 34, 33 (about 7 GB)."""
    from pentago_b200 import sweep
    from pentago_b200.end import section_sig
    res = sweep.sweep(section_sig([[4, 4], [5, 4], [4, 5], [4, 3]]))
    assert sorted(res) == [33, 34, 35]
    check_golden(res)


def test_sweep_single_quadrant_root_matches_golden_counts(cuda):
    """Root [[5,4],[5,4],[4,5],[2,3]] (32 stones): a chain along quadrant 3."""
    from pentago_b200 import sweep
    from pentago_b200.end import section_sig
    res = sweep.sweep(section_sig([[5, 4], [5, 4], [4, 5], [2, 3]]))
    assert sorted(res) == [32, 33, 34, 35]
    check_golden(res)


def test_slice35_sections_match_golden_counts(cuda):
    """A few whole 35-stone sections, computed directly (no children)."""
    import torch
    from pentago_b200 import capi, sweep
    sigs = np.sort(GOLD["counts_35"][:, 0][::37].copy())
    off = sweep.slice_layout(sigs)
    assert off[-1] * 64 < 4e9
    t = torch.empty((int(off[-1]), 8), dtype=torch.int64, device=cuda)
    L = capi.lib()
    s = capi.stream_handle()
    capi.check(L.pg_end_sweep_slice(capi.ptr(sigs), len(sigs), t.data_ptr(), None, 0, None, s))
    counts = torch.zeros((len(sigs), 3), dtype=torch.int64, device=cuda)
    capi.check(L.pg_section_counts(capi.ptr(sigs), len(sigs), t.data_ptr(), counts.data_ptr(), s))
    check_golden({35: sweep.to_golden(sigs, counts.cpu().numpy().view(np.uint64), 35)})


def test_config2_root_sweep_matches_golden_counts(cuda):
    """The full in-core sweep below root [[4,4],[4,5],[4,3],[3,3]]: slices
    35 -> 30 (39 sections, 141.7 GB at the peak pair), every section's counts
    equal to the original solve's (data/counts-30..35.npy)."""
    import torch
    from pentago_b200 import sweep
    from pentago_b200.end import section_sig
    free = torch.cuda.mem_get_info()[0]
    if free < 150e9:
        pytest.skip(f"needs about 142 GB of free device memory, {free / 1e9:.1f} GB free")
    res = sweep.sweep(section_sig([[4, 4], [4, 5], [4, 3], [3, 3]]))
    assert sorted(res) == [30, 31, 32, 33, 34, 35]
    assert [len(res[s]) for s in range(30, 36)] == [1, 3, 8, 10, 10, 7]
    check_golden(res)


HIGH = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "high_samples.json")))


def disk_supers(node, turn):
    """An end-engine node [we win, we win or tie] as the on-disk pair [black
    wins, white wins] (pentago/end/check.cc:154-156, 197-200)."""
    win, notlost = node[:4], node[4:]
    pair = [win, ~notlost]
    return pair[::-1] if turn else pair


@pytest.mark.parametrize("slice_", [35, 34, 33])
def test_high_samples_match_swept_sections(cuda, O, slice_):
    """The 32 samples of pentago/high/high_test.cc:41-85 for one slice: boards
    with both sides' full rotation sets from the 2013 solve.  Each board's
    section is swept as a root (its slice and every slice below it), the
    board's node is read from the root's slice tensor, mapped back to the
    board by the board's symmetry, and both 256-rotation supers must equal the
    sample's (the reference test checks one rotation per board)."""
    import ctypes
    from pentago_b200 import sweep
    from pentago_b200.end import section_shape
    boards = HIGH[str(slice_)]["boards"]
    wins = np.array(HIGH[str(slice_)]["wins"], np.uint64).reshape(-1, 2, 4)
    groups = {}
    for i, b in enumerate(boards):
        sec, turn, sym = ctypes.c_uint64(), ctypes.c_int32(), ctypes.c_uint16()
        idx = (ctypes.c_int32 * 4)()
        O.lookup_locate(ctypes.c_uint64(b), ctypes.byref(sec), idx, ctypes.byref(sym), ctypes.byref(turn))
        groups.setdefault(sec.value, []).append((i, list(idx), sym.value, turn.value))
    checked = 0
    for sec, items in groups.items():
        res, tensor, sigs = sweep.sweep(sec, keep_last=True)
        assert min(res) == slice_ and list(sigs) == [sec]
        shape = section_shape(sec)
        for i, idx, sym, turn in items:
            b = [q // 8 for q in idx]
            bs = [min(8, shape[q] - 8 * b[q]) for q in range(4)]
            off, before = 0, 1
            for q in range(4):
                after = int(np.prod(shape[q + 1:]))
                off += before * 8 * b[q] * after
                before *= bs[q]
            inner = (((idx[0] % 8) * bs[1] + idx[1] % 8) * bs[2] + idx[2] % 8) * bs[3] + idx[3] % 8
            node = tensor[off + inner].cpu().numpy().view(np.uint64)
            for side, s in enumerate(disk_supers(node, turn)):
                got = np.zeros(4, np.uint64)
                O.transform_super(P(np.array([sym], np.uint16)), P(np.ascontiguousarray(s)), P(got), 1)
                assert np.array_equal(got, wins[i, side]), f"slice {slice_} board {boards[i]} side {side}"
            checked += 1
        del tensor
    assert checked == 32
