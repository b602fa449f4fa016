"""Learned rANS (format 3) on the GPU, against the CPU oracle of the format:
the coder's integer frequencies and stream bytes equal the oracle's, the
training gradient matches the oracle's, decoding is lossless, and a network
trained by the library's own kernels codes real solved blocks at least 10%
smaller than the format-2 static coder it falls back to."""
import ctypes
import functools

import numpy as np
import pytest

from tests.oracle import P

pytestmark = pytest.mark.gpu

ROOT = [[4, 4], [5, 4], [4, 5], [4, 3]]   # a 33-stone section: slices 35..33 solved in seconds


@functools.lru_cache(maxsize=1)
def solved():
    """Blocks of the solved root slice: refs, node offsets, node counts, slice tensor."""
    import torch
    from pentago_b200 import capi, learned, sweep
    from pentago_b200.end import section_sig
    capi.check(capi.lib().pg_init())
    _, slice_t, sigs = sweep.sweep(section_sig(ROOT), keep_last=True)
    refs, off, nodes = learned.slice_blocks(sigs, sweep.slice_layout(sigs))
    torch.cuda.synchronize()
    return refs, off, nodes, slice_t


def pick(idx):
    from pentago_b200 import learned
    refs, off, nodes, slice_t = solved()
    idx = np.asarray(idx)
    sym, offsets = learned.block_symbols(slice_t, off[idx], nodes[idx], 33 & 1)
    return learned.subset(refs, idx), sym, offsets, nodes[idx]


def edge_and_full():
    """One full block and the last block of the grid (ragged)."""
    _, _, nodes, _ = solved()
    full = int(np.nonzero(nodes == 4096)[0][0])
    return [full, len(nodes) - 1]


def random_model(seed, scale):
    from pentago_b200 import capi, learned
    rng = np.random.default_rng(seed)
    params = (rng.standard_normal(learned.N_PARAMS) * scale).astype(np.float32)
    model = np.zeros(learned.model_bytes(), np.uint8)
    capi.check(capi.lib().pg_learned_export(P(params), P(model)))
    return params, model.tobytes()


@functools.lru_cache(maxsize=1)
def trained():
    """A model trained on 1% of the slice's blocks (seeded), with its trainer."""
    from pentago_b200 import learned
    _, _, nodes, _ = solved()
    rng = np.random.default_rng(5)
    tb = np.sort(rng.choice(len(nodes), max(8, len(nodes) // 100), replace=False))
    refs, sym, offsets, n = pick(tb)
    tr = learned.Trainer(refs, sym, offsets, n, seed=3)
    hist = tr.run(400, batch=16384, log_every=100)
    return tr.model(), hist, set(tb.tolist())


def oracle_stream(O, model, ref, sym):
    blk = np.array(list(ref.block), np.int32)
    out = np.zeros(200 + 512 * (sym.size // 256), np.uint8)
    mbytes = np.frombuffer(model, np.uint8)
    n = O.lm_encode(P(mbytes), ref.section, P(blk), P(sym), P(out), out.size)
    assert n > 0
    st = np.zeros(sym.size // 4 + 1000, np.uint8)
    m = O.rans_encode(P(sym), sym.size, P(st), st.size)
    assert m > 0
    return out[:n].tobytes(), st[:m].tobytes()


def test_freqs_match_oracle(cuda, O):
    import torch
    from pentago_b200 import learned
    refs, sym, offsets, nodes = pick(edge_and_full())
    host = sym.cpu().numpy()
    off = offsets.cpu().numpy()
    for seed, scale in ((1, 0.05), (2, 0.3), (3, 2.0)):
        _, model = random_model(seed, scale)
        rng = np.random.default_rng(seed)
        for s in range(len(refs)):
            k = 3000
            samples = (np.int64(s) << 24) | (rng.integers(0, nodes[s], k).astype(np.int64) << 8) | rng.integers(0, 256, k)
            got = learned.freqs(model, refs, sym, offsets, torch.from_numpy(samples).cuda()).cpu().numpy()
            want = np.zeros((k, 3), np.uint32)
            blk = np.array(list(refs[s].block), np.int32)
            local = np.ascontiguousarray(samples & 0xffffff)
            # (arrays handed to the oracle by address are kept in variables while it runs)
            mbytes = np.frombuffer(model, np.uint8)
            block_sym = np.ascontiguousarray(host[off[s]:off[s + 1]])
            assert O.lm_freqs(P(mbytes), refs[s].section, P(blk), P(block_sym), P(local), k, P(want)) == 0
            assert np.array_equal(got.astype(np.uint32), want)


def test_streams_match_oracle_bytes(cuda, O):
    from pentago_b200 import learned
    refs, sym, offsets, nodes = pick(edge_and_full())
    host = sym.cpu().numpy()
    off = offsets.cpu().numpy()
    for model in (trained()[0], random_model(4, 0.3)[1]):
        data, doff, dsz = learned.encode(model, refs, sym, offsets, nodes)
        data, doff, dsz = data.cpu().numpy(), doff.cpu().numpy(), dsz.cpu().numpy()
        for s in range(len(refs)):
            lm, st = oracle_stream(O, model, refs[s], np.ascontiguousarray(host[off[s]:off[s + 1]]))
            got = data[doff[s]:doff[s] + dsz[s]].tobytes()
            assert got == (lm if len(lm) < len(st) else st)


def test_gradient_matches_oracle(cuda, O):
    import torch
    from pentago_b200 import learned
    refs, sym, offsets, nodes = pick(edge_and_full()[:1])
    rng = np.random.default_rng(8)
    params = (rng.standard_normal(learned.N_PARAMS) * 0.2).astype(np.float32)
    k = 5000
    local = (rng.integers(0, nodes[0], k).astype(np.int64) << 8) | rng.integers(0, 256, k)
    tr = learned.Trainer(refs, sym, offsets, nodes, params=torch.from_numpy(params).cuda())
    g, loss = tr.grad_of(torch.from_numpy(local).cuda())
    g = g.cpu().numpy().astype(np.float64)
    want = np.zeros(learned.N_PARAMS)
    blk = np.array(list(refs[0].block), np.int32)
    host = sym.cpu().numpy()
    wl = O.lm_grad(P(params), refs[0].section, P(blk), P(host), P(local), k, P(want))
    assert abs(float(loss.item()) - wl) <= 1e-4 * abs(wl)
    scale = np.abs(want).max()
    assert np.abs(g - want).max() <= 2e-4 * scale
    # every parameter block receives gradient
    for a, b in ((learned.P_W1, learned.P_B1), (learned.P_W2, learned.P_B2), (learned.P_W3, learned.P_B3)):
        assert np.abs(want[a:b]).max() > 0


def test_trained_model_beats_static_and_roundtrips(cuda):
    import torch
    from pentago_b200 import learned
    model, hist, train_blocks = trained()
    assert hist[-1][1] < hist[0][1]
    _, _, nodes, _ = solved()
    rng = np.random.default_rng(6)
    held_out = [i for i in rng.choice(len(nodes), 96, replace=False) if i not in train_blocks][:64]
    refs, sym, offsets, n = pick(sorted(held_out))
    data, doff, dsz = learned.encode(model, refs, sym, offsets, n)
    static = learned.static_sizes(sym, offsets)
    learned_bytes, static_bytes = int(dsz.sum().item()), int(static.sum().item())
    assert learned_bytes <= 0.9 * static_bytes, (learned_bytes, static_bytes)
    back, _, status = learned.decode(model, refs, data, doff, dsz, n)
    assert (status.cpu().numpy() == n * 256).all()
    assert torch.equal(back, sym)


def test_network_gain_on_held_out_blocks(cuda):
    """The same 64 held-out blocks coded three ways: format 2 (one order-0
    table per block), the store coder's counted context table (the same kind
    of context as the network's neighbour and previous-node features, counted
    from the blocks themselves, no network) and the trained network.  Prints
    the three figures in bits per position; the network must be at least 10%
    smaller than format 2, smaller than the counted table, and round-trip
    (the store coder's own round trips are tested with the compressed
    sweeps)."""
    import torch
    from pentago_b200 import learned
    model, _, train_blocks = trained()
    refs_all, off_all, nodes_all, slice_t = solved()
    rng = np.random.default_rng(6)
    held_out = sorted([i for i in rng.choice(len(nodes_all), 96, replace=False) if i not in train_blocks][:64])
    refs, sym, offsets, n = pick(held_out)
    data, doff, dsz = learned.encode(model, refs, sym, offsets, n)
    back, _, status = learned.decode(model, refs, data, doff, dsz, n)
    assert torch.equal(back, sym)
    static, _, _, ok = learned.static_roundtrip(sym, offsets)
    assert ok
    ctx_sizes, table_bytes = learned.store_sizes(slice_t, off_all[held_out], nodes_all[held_out], 33 & 1)
    positions = int(sym.numel())
    bits = {"static": 8.0 * int(static.sum().item()) / positions,
            "context_table": 8.0 * (int(ctx_sizes.sum()) + table_bytes) / positions,
            "learned": 8.0 * int(dsz.sum().item()) / positions}
    print("bits per position on held-out blocks:", bits)
    assert bits["learned"] <= 0.9 * bits["static"], bits
    assert bits["context_table"] < bits["static"], bits
    assert bits["learned"] < bits["context_table"], bits


def test_untrained_model_falls_back_to_static(cuda):
    import torch
    from pentago_b200 import learned
    refs, sym, offsets, nodes = pick(edge_and_full())
    zero = learned.export(torch.zeros(learned.N_PARAMS))   # uniform: 1.58 bits per symbol
    data, doff, dsz = learned.encode(zero, refs, sym, offsets, nodes)
    static = learned.static_sizes(sym, offsets)
    assert torch.equal(dsz, static)
    d = data.cpu().numpy()
    for s in range(len(refs)):
        assert d[int(doff[s]):int(doff[s]) + 4].tobytes() == (2).to_bytes(4, "little")
    back, _, status = learned.decode(zero, refs, data, doff, dsz, nodes)
    assert torch.equal(back, sym)


def test_decoder_rejects_bad_streams(cuda):
    from pentago_b200 import capi, learned
    model = trained()[0]
    refs, sym, offsets, nodes = pick(edge_and_full())
    data, doff, dsz = learned.encode(model, refs, sym, offsets, nodes)
    d = data.cpu().numpy()
    assert all(d[int(doff[s]):int(doff[s]) + 4].tobytes() == (3).to_bytes(4, "little") for s in range(len(refs)))
    # another model
    _, other = random_model(9, 0.1)
    _, _, status = learned.decode(other, refs, data, doff, dsz, nodes)
    assert (status.cpu().numpy() == capi.PG_ERR_FORMAT).all()
    # truncated, and one word short
    for cut in (100, 2):
        _, _, status = learned.decode(model, refs, data, doff, dsz - cut, nodes)
        assert (status.cpu().numpy() == capi.PG_ERR_FORMAT).all()
    # a flipped word in the middle: decoding runs to the end and fails the final-state check
    bad = data.clone()
    mid = int(doff[0]) + 148 + 2 * ((int(dsz[0]) - 148) // 4)
    bad[mid] ^= 0x5A
    back, _, status = learned.decode(model, refs, bad, doff, dsz, nodes)
    assert status.cpu().numpy()[0] == capi.PG_ERR_FORMAT
    assert status.cpu().numpy()[1] == nodes[1] * 256
