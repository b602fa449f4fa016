"""Slice sweeps on the GPU against the reference's golden per-section counts
(data/counts-N.npy from the original solve) and against per-line compute."""
import os

import numpy as np
import pytest

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
