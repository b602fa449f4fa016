"""The store coder's CPU restatement (oracle/store_oracle.c): its own round
trip on ragged blocks in both turns, blocks stored raw, damaged streams
refused, and its bound equal to the library's."""
import numpy as np
import pytest

from tests.oracle import P

COUNTS = [1, 7, 31, 32, 33, 100, 511, 512, 4095, 4096]


def skewed_nodes(n, seed):
    """Nodes whose rotations are correlated the way solved ones are: runs of
    equal words, so the contexts matter."""
    rng = np.random.default_rng(seed)
    x = rng.integers(0, 2**64 - 1, size=(n, 4), dtype=np.uint64, endpoint=True)
    win = x & rng.integers(0, 2**64 - 1, size=(n, 4), dtype=np.uint64, endpoint=True) & \
        rng.integers(0, 2**64 - 1, size=(n, 4), dtype=np.uint64, endpoint=True)
    nl = win | (x & rng.integers(0, 2**64 - 1, size=(n, 4), dtype=np.uint64, endpoint=True))
    nodes = np.concatenate([win, nl], 1)
    nodes[1::3] = nodes[0::3][:len(nodes[1::3])]   # repeated neighbours
    return np.ascontiguousarray(nodes)


def batch(counts, seed):
    counts = np.array(counts, np.int32)
    first = np.concatenate([[0], np.cumsum(counts)[:-1]]).astype(np.int64)
    return skewed_nodes(int(counts.sum()), seed), first, counts


@pytest.mark.parametrize("turn", [0, 1])
def test_store_oracle_round_trip(O, turn):
    nodes, first, counts = batch(COUNTS, 11 + turn)
    table = np.zeros(3072, np.uint16)
    O.store_table(P(nodes), P(first), P(counts), len(counts), turn, P(table))
    f = table.reshape(1024, 3).astype(np.int64)
    assert (f >= 1).all() and (f.sum(1) == 1 << 14).all()
    raw = 0
    for b, n in enumerate(counts.tolist()):
        block = np.ascontiguousarray(nodes[first[b]:first[b] + n])
        out = np.zeros(int(O.store_bound(n)), np.uint8)
        size = O.store_encode_block(P(block), n, turn, P(table), P(out))
        assert 128 < size <= O.store_bound(n)
        raw += size == 128 + 64 * n
        back = np.zeros_like(block)
        assert O.store_decode_block(P(out), size, n, turn, P(table), P(back)) == n
        assert np.array_equal(back, block), (b, n)
        if n >= 100:
            bad = out.copy()
            bad[128 + (size - 128) // 2] ^= 0x5A
            assert O.store_decode_block(P(bad), size, n, turn, P(table), P(back)) == -1
            assert O.store_decode_block(P(out), size - 1, n, turn, P(table), P(back)) == -1
    assert raw < len(counts)   # the skewed blocks compress


def test_store_oracle_raw_blocks(O):
    """Nodes with no structure cannot be coded within their raw size: they are
    stored raw and come back unchanged."""
    rng = np.random.default_rng(3)
    n = 4096
    a = rng.integers(0, 2**64 - 1, size=(n, 4), dtype=np.uint64, endpoint=True)
    b = rng.integers(0, 2**64 - 1, size=(n, 4), dtype=np.uint64, endpoint=True)
    nodes = np.ascontiguousarray(np.concatenate([a & b, a | b], 1))
    skew, _, _ = batch([n], 5)
    table = np.zeros(3072, np.uint16)
    first, counts = np.zeros(1, np.int64), np.array([n], np.int32)
    O.store_table(P(skew), P(first), P(counts), 1, 0, P(table))
    out = np.zeros(int(O.store_bound(n)), np.uint8)
    size = O.store_encode_block(P(nodes), n, 0, P(table), P(out))
    assert size == 128 + 64 * n and (out[:4] == 0xff).all() and not out[4:128].any()
    back = np.zeros_like(nodes)
    assert O.store_decode_block(P(out), size, n, 0, P(table), P(back)) == n
    assert np.array_equal(back, nodes)


def test_store_oracle_bound_matches_library(O):
    from pentago_b200 import capi
    L = capi.lib()
    for n in [0, 1, 31, 32, 33, 1000, 4096]:
        assert O.store_bound(n) == L.pg_store_bound(n)
