"""Slices kept compressed in HBM: symbols back to nodes, the store coder's
round trip on ragged blocks of random nodes and its refusal of damaged
streams, a solved slice through the per-block store and back, and a sweep
that keeps every
finished slice compressed, computing each slice one child section at a time,
with the same counts and the same last slice as the plain sweep; and a root
too deep to sweep raw in one device's memory, solved compressed and checked
against the reference's counts."""
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


def test_store_coder_roundtrip_and_damage(cuda):
    import torch
    from pentago_b200 import capi
    from pentago_b200.slice_store import HEAD, store_bound
    L = capi.lib()
    counts = np.array([1, 7, 8, 9, 100, 4096, 4095, 512], np.int32)
    assert [L.pg_store_bound(int(c)) for c in counts] == store_bound(counts).tolist()
    first = np.concatenate([[0], np.cumsum(counts)[:-1]]).astype(np.int64)
    n = int(counts.sum())
    g = torch.Generator(device="cuda")
    g.manual_seed(5)
    r = lambda: torch.randint(-2**63, 2**63 - 1, (n, 4), dtype=torch.int64, device="cuda", generator=g)
    x = r()
    win = x & r() & r()             # skewed, so the contexts matter
    nodes = torch.cat([win, win | (x & r())], 1).contiguous()
    t = lambda a, dt=np.int64: torch.from_numpy(np.ascontiguousarray(a, dtype=dt)).cuda()
    d_first, d_count = t(first), t(counts, np.int32)
    for turn in (0, 1):
        table = torch.empty(3072, dtype=torch.int16, device="cuda")
        capi.check(L.pg_store_table(nodes.data_ptr(), d_first.data_ptr(), d_count.data_ptr(), len(counts), turn,
                                    table.data_ptr(), None))
        f = table.cpu().numpy().view(np.uint16).reshape(1024, 3).astype(np.int64)
        assert (f >= 1).all() and (f.sum(1) == 1 << 14).all()
        caps = store_bound(counts)
        off = np.concatenate([[0], np.cumsum(caps)[:-1]]).astype(np.int64)
        out = torch.zeros(int(caps.sum()), dtype=torch.uint8, device="cuda")
        sizes = torch.zeros(len(counts), dtype=torch.int64, device="cuda")
        d_off = t(off)
        capi.check(L.pg_store_encode(nodes.data_ptr(), d_first.data_ptr(), d_count.data_ptr(), len(counts), turn,
                                     table.data_ptr(), out.data_ptr(), d_off.data_ptr(), sizes.data_ptr(), None))
        sz = sizes.cpu().numpy()
        assert (sz > HEAD).all() and (sz <= caps).all()

        def decode(data, sizes_):
            back = torch.zeros_like(nodes)
            status = torch.zeros(len(counts), dtype=torch.int64, device="cuda")
            capi.check(L.pg_store_decode(data.data_ptr(), d_off.data_ptr(), t(sizes_).data_ptr(), d_count.data_ptr(),
                                         d_first.data_ptr(), len(counts), turn, table.data_ptr(), back.data_ptr(),
                                         status.data_ptr(), None))
            return back, status.cpu().numpy()
        back, status = decode(out, sz)
        assert status.tolist() == counts.tolist() and torch.equal(back, nodes)
        # blocks that no lane can code within their raw size are stored raw
        noise = torch.randint(-2**63, 2**63 - 1, (n, 8), dtype=torch.int64, device="cuda", generator=g)
        noisy = torch.cat([noise[:, :4] & noise[:, 4:], noise[:, :4] | noise[:, 4:]], 1).contiguous()
        raw_sizes = torch.zeros(len(counts), dtype=torch.int64, device="cuda")
        raw_out = torch.zeros_like(out)
        capi.check(L.pg_store_encode(noisy.data_ptr(), d_first.data_ptr(), d_count.data_ptr(), len(counts), turn,
                                     table.data_ptr(), raw_out.data_ptr(), d_off.data_ptr(), raw_sizes.data_ptr(),
                                     None))
        rs = raw_sizes.cpu().numpy()
        assert (rs <= caps).all() and (rs == HEAD + 64 * counts.astype(np.int64)).any()
        back = torch.zeros_like(noisy)
        status = torch.zeros(len(counts), dtype=torch.int64, device="cuda")
        capi.check(L.pg_store_decode(raw_out.data_ptr(), d_off.data_ptr(), t(rs).data_ptr(), d_count.data_ptr(),
                                     d_first.data_ptr(), len(counts), turn, table.data_ptr(), back.data_ptr(),
                                     status.data_ptr(), None))
        assert status.cpu().numpy().tolist() == counts.tolist() and torch.equal(back, noisy)
        bad = out.clone()
        bad[int(off[5]) + 40 + int(sz[5]) // 2] ^= 0x5A   # the middle of the 4096-node block
        _, status = decode(bad, sz)
        assert status[5] == capi.PG_ERR_FORMAT and status[4] == counts[4]
        _, status = decode(out, sz - 1)                    # every stream one byte short
        assert (status == capi.PG_ERR_FORMAT).all()


def test_compressed_slice_roundtrip(cuda):
    import torch
    from pentago_b200 import sweep
    from pentago_b200.end import section_sig
    from pentago_b200.slice_store import compressed_slice
    _, nodes, sigs = sweep.sweep(section_sig(ROOT), min_slice=34, keep_last=True)
    store = compressed_slice(nodes, sigs, 34 & 1, chunk_nodes=1 << 20)
    assert len(store.chunks) > 1 and store.bytes < store.raw_bytes / 2.5
    for i in range(len(sigs)):
        assert torch.equal(store.section_nodes(i), nodes[int(store.base[i]):int(store.base[i + 1])])


def test_compressed_sweep_matches_plain(cuda, tmp_path):
    import torch
    from pentago_b200 import supertensor, sweep
    from pentago_b200.end import section_sig
    root = section_sig(ROOT)
    plain, last, _ = sweep.sweep(root, keep_last=True)
    timings = {}
    packed, last2, _ = sweep.sweep(root, keep_last=True, compress=True, timings=timings, checkpoint=str(tmp_path),
                                   level=1)
    assert sorted(plain) == sorted(packed)
    for s in plain:
        assert np.array_equal(plain[s], packed[s]), s
    assert torch.equal(last, last2)
    assert all(timings[s]["compressed_bytes"] < timings[s]["raw_bytes"] / 2.5 for s in (35, 34))
    # the section-by-section checkpoint holds the same slice
    _, _, back = supertensor.read_slice(str(tmp_path / "slice-33.pentago"))
    assert torch.equal(back, last)


# A 28-stone root whose slices 31 and 30 (105.4 + 99.5 GB) do not fit a B200's
# HBM side by side raw (tests/golden/make_golden.py: DEEP_ROOT).
DEEP_ROOT = [[4, 4], [4, 5], [4, 3], [2, 2]]


def test_deep_root_needs_compression_and_matches_golden(cuda):
    """The plain sweep of the 28-stone root is refused before it allocates
    anything; the compressed sweep solves slices 35 down to 28 well inside the
    device's memory, and every one of the 75 sections' counts equals the row
    of data/counts-N.npy from the original solve (about two minutes)."""
    import os
    import torch
    from pentago_b200 import capi, sweep
    from pentago_b200.end import section_sig
    here = os.path.join(os.path.dirname(__file__), "golden")
    gold = dict(np.load(os.path.join(here, "counts_30_35.npz")))
    gold.update(dict(np.load(os.path.join(here, "counts_28_29.npz"))))
    root = section_sig(DEEP_ROOT)
    with pytest.raises(capi.PentagoError) as refused:
        sweep.sweep(root)
    assert refused.value.code == capi.PG_ERR_CAPACITY
    torch.cuda.empty_cache()
    torch.cuda.reset_peak_memory_stats()
    res = sweep.sweep(root, compress=True)
    assert sorted(res) == list(range(28, 36))
    assert sum(len(rows) for rows in res.values()) == 75
    for s, rows in res.items():
        want = {int(r[0]): r for r in gold[f"counts_{s}"]}
        for r in rows:
            assert np.array_equal(want[int(r[0])], r), f"slice {s} section {int(r[0]):#x}"
    total = torch.cuda.get_device_properties(0).total_memory
    assert torch.cuda.max_memory_allocated() < 0.75 * total


def test_store_coder_matches_oracle_bytes(cuda, O):
    """The GPU's frequency table and every stream byte equal the CPU
    restatement's (oracle/store_oracle.c): skewed random blocks of ragged
    sizes in both turns, a batch of 2,100 small blocks (the table then counts
    every second block), and full blocks of a solved slice."""
    import torch
    from pentago_b200 import capi, sweep
    from pentago_b200.end import section_sig
    from pentago_b200.slice_store import slice_blocks, store_bound
    from tests.oracle import P
    from tests.test_store_cpu import COUNTS, batch
    L = capi.lib()
    t = lambda a, dt=np.int64: torch.from_numpy(np.ascontiguousarray(a, dtype=dt)).cuda()

    def check(nodes_np, first, counts, turn, blocks):
        dev = torch.from_numpy(nodes_np.view(np.int64)).cuda()
        d_first, d_count = t(first), t(counts, np.int32)
        table = torch.empty(3072, dtype=torch.int16, device="cuda")
        capi.check(L.pg_store_table(dev.data_ptr(), d_first.data_ptr(), d_count.data_ptr(), len(counts), turn,
                                    table.data_ptr(), None))
        want_table = np.zeros(3072, np.uint16)
        O.store_table(P(nodes_np), P(first), P(counts), len(counts), turn, P(want_table))
        assert np.array_equal(table.cpu().numpy().view(np.uint16), want_table)
        caps = store_bound(counts)
        off = np.concatenate([[0], np.cumsum(caps)[:-1]]).astype(np.int64)
        out = torch.zeros(int(caps.sum()), dtype=torch.uint8, device="cuda")
        sizes = torch.zeros(len(counts), dtype=torch.int64, device="cuda")
        d_off = t(off)
        capi.check(L.pg_store_encode(dev.data_ptr(), d_first.data_ptr(), d_count.data_ptr(), len(counts), turn,
                                     table.data_ptr(), out.data_ptr(), d_off.data_ptr(), sizes.data_ptr(), None))
        host, sz = out.cpu().numpy(), sizes.cpu().numpy()
        for b in blocks:
            n = int(counts[b])
            block = np.ascontiguousarray(nodes_np[first[b]:first[b] + n])
            want = np.zeros(int(O.store_bound(n)), np.uint8)
            size = O.store_encode_block(P(block), n, turn, P(want_table), P(want))
            assert sz[b] == size, (b, n, turn)
            assert np.array_equal(host[off[b]:off[b] + size], want[:size]), (b, n, turn)

    for turn in (0, 1):
        nodes, first, counts = batch(COUNTS, 21 + turn)
        check(nodes, first, counts, turn, range(len(counts)))
    rng = np.random.default_rng(4)
    nodes, first, counts = batch(rng.integers(1, 9, 2100).tolist(), 8)
    check(nodes, first, counts, 1, rng.choice(2100, 40, replace=False))
    _, slice_t, sigs = sweep.sweep(section_sig(ROOT), min_slice=34, keep_last=True)
    _, bfirst, bcount, _, _ = slice_blocks(sigs)
    full = np.nonzero(bcount == 4096)[0][:16]
    lo, hi = int(bfirst[full[0]]), int(bfirst[full[-1]]) + 4096
    nodes = np.ascontiguousarray(slice_t[lo:hi].cpu().numpy().view(np.uint64))
    check(nodes, (bfirst[full] - lo).astype(np.int64), bcount[full].astype(np.int32), 0, range(len(full)))
