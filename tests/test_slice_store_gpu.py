"""Slices kept compressed in HBM: symbols back to nodes, a solved slice
through the per-block format-2 store and back, and a sweep that keeps every
finished slice compressed, computing each slice one child section at a time,
with the same counts and the same last slice as the plain sweep."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = [[4, 4], [5, 4], [4, 5], [4, 3]]


def test_symbols_to_nodes_inverts_node_symbols(cuda):
    import torch
    from pentago_b200 import capi, rans
    g = torch.Generator(device="cuda")
    g.manual_seed(3)
    r = lambda: torch.randint(-2**63, 2**63 - 1, (10007, 4), dtype=torch.int64, device="cuda", generator=g)
    win = r() & r()
    nodes = torch.cat([win, win | r()], 1).contiguous()   # win within not-lost
    for turn in (0, 1):
        sym = rans.node_symbols(nodes, turn)
        back = torch.empty_like(nodes)
        capi.check(capi.lib().pg_symbols_nodes(sym.data_ptr(), nodes.shape[0], turn, back.data_ptr(), None))
        assert torch.equal(back, nodes)


def test_compressed_slice_roundtrip(cuda):
    import torch
    from pentago_b200 import sweep
    from pentago_b200.end import section_sig
    from pentago_b200.slice_store import compressed_slice
    _, nodes, sigs = sweep.sweep(section_sig(ROOT), min_slice=34, keep_last=True)
    store = compressed_slice(nodes, sigs, 34 & 1, chunk_nodes=1 << 20)
    assert len(store.chunks) > 1 and store.bytes < store.raw_bytes / 1.3
    for i in range(len(sigs)):
        assert torch.equal(store.section_nodes(i), nodes[int(store.base[i]):int(store.base[i + 1])])


def test_compressed_sweep_matches_plain(cuda):
    import torch
    from pentago_b200 import sweep
    from pentago_b200.end import section_sig
    root = section_sig(ROOT)
    plain, last, _ = sweep.sweep(root, keep_last=True)
    timings = {}
    packed, last2, _ = sweep.sweep(root, keep_last=True, compress=True, timings=timings)
    assert sorted(plain) == sorted(packed)
    for s in plain:
        assert np.array_equal(plain[s], packed[s]), s
    assert torch.equal(last, last2)
    assert all(timings[s]["compressed_bytes"] < timings[s]["raw_bytes"] / 1.3 for s in (35, 34))
