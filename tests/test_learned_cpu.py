"""Learned rANS (format 3) on the CPU: the oracle's coder round-trips and
rejects streams of another model, its frequency tables are valid, and the
library's model serialization is the specified one (bf16, round to nearest
even; the layer-2 weights on their column grids)."""
import ctypes

import numpy as np
import pytest

from tests.oracle import P

SIG = None


def section(counts):
    from pentago_b200.end import section_sig
    return section_sig(counts)


def random_model(seed, scale=0.1):
    from pentago_b200 import capi, learned
    rng = np.random.default_rng(seed)
    params = (rng.standard_normal(learned.N_PARAMS) * scale).astype(np.float32)
    model = np.zeros(learned.model_bytes(), np.uint8)
    capi.check(capi.lib().pg_learned_export(P(params), P(model)))
    return params, model


def block_symbols(n, seed):
    """Correlated ternaries: most rotations of a node share its value."""
    rng = np.random.default_rng(seed)
    base = rng.integers(0, 3, size=(n, 1))
    return np.where(rng.random((n, 256)) < 0.85, base, rng.integers(0, 3, size=(n, 256))).astype(np.uint8)


def encode(O, model, sig, blk, sym):
    out = np.zeros(200 + 512 * (sym.size // 256), np.uint8)
    n = O.lm_encode(P(model), sig, P(blk), P(sym), P(out), out.size)
    assert n > 0
    return out[:n]


@pytest.mark.parametrize("counts,block", [
    ([[2, 2], [2, 1], [1, 2], [2, 2]], [0, 0, 1, 0]),   # full block, 4096 nodes
    ([[1, 1], [0, 0], [0, 1], [1, 0]], [0, 0, 0, 0]),   # small block (72 x 1 x 9 x 9)
])
def test_oracle_roundtrip(O, counts, block):
    sig = section(counts)
    blk = np.array(block, np.int32)
    n = O.lm_nodes(sig, P(blk))
    assert n > 0
    _, model = random_model(1)
    sym = block_symbols(n, 2)
    data = encode(O, model, sig, blk, sym)
    dec = np.zeros(256 * n, np.uint8)
    assert O.lm_decode(P(model), sig, P(blk), P(data), data.size, P(dec), dec.size) == 256 * n
    assert np.array_equal(dec.reshape(n, 256), sym)
    # another model, a truncated stream, a stream of another block: rejected
    _, other = random_model(3)
    assert O.lm_decode(P(other), sig, P(blk), P(data), data.size, P(dec), dec.size) < 0
    assert O.lm_decode(P(model), sig, P(blk), P(data), data.size - 2, P(dec), dec.size) < 0


def test_oracle_freqs_are_valid_tables(O):
    sig = section([[2, 2], [2, 1], [1, 2], [2, 2]])
    blk = np.array([0, 0, 1, 0], np.int32)
    n = O.lm_nodes(sig, P(blk))
    sym = block_symbols(n, 5)
    for scale in (0.01, 0.5, 8.0):   # nearly uniform to extremely confident
        _, model = random_model(7, scale)
        rng = np.random.default_rng(11)
        samples = (rng.integers(0, n, 2000).astype(np.int64) << 8) | rng.integers(0, 256, 2000)
        f = np.zeros((2000, 3), np.uint32)
        assert O.lm_freqs(P(model), sig, P(blk), P(sym), P(samples), 2000, P(f)) == 0
        assert (f.sum(1) == 32768).all() and (f >= 1).all()


def test_export_format(O):
    from pentago_b200 import capi, learned
    params = np.array([1.0, -2.5, 1.00390625, 1.01171875, 3.0e38] + [0.0] * (learned.N_PARAMS - 5), np.float32)
    # W2 column 0: largest magnitude 1.0 = 0.5 2^1, so its grid is 2^-6
    for k, w in ((0, 1.0), (1, 0.3), (2, -0.0123), (3, 0.5078125)):
        params[learned.P_W2 + 64 * k] = w
    model = np.zeros(learned.model_bytes(), np.uint8)
    assert learned.model_bytes() == 12 + 2 * learned.N_PARAMS
    capi.check(capi.lib().pg_learned_export(P(params), P(model)))
    assert model[:4].tobytes() == b"PGLM"
    assert np.frombuffer(model[4:12].tobytes(), np.uint32).tolist() == [3, learned.N_PARAMS]
    h = np.frombuffer(model[12:].tobytes(), np.uint16)
    # 1.00390625 = 1 + 2^-8 is a tie and rounds to even (1.0); 1 + 3 * 2^-8 rounds up
    assert h[:4].tolist() == [0x3F80, 0xC020, 0x3F80, 0x3F82]
    # 0.3 -> 19/64, -0.0123 -> -1/64, 0.5078125 = 32.5/64 -> 32/64 (tie to even)
    col = [h[learned.P_W2 + 64 * k] for k in range(4)]
    assert col == [0x3F80, 0x3E98, 0xBC80, 0x3F00]
    bad = params.copy()
    bad[7] = np.nan
    assert capi.lib().pg_learned_export(P(bad), P(model)) == capi.PG_ERR_ARG
    # the oracle takes the exported model, and refuses version 1 and a W2 off its grid
    sig = section([[2, 2], [2, 1], [1, 2], [2, 2]])
    blk = np.array([0, 0, 1, 0], np.int32)
    n = O.lm_nodes(sig, P(blk))
    sym = block_symbols(n, 5)
    out = np.zeros(200 + 512 * n, np.uint8)
    assert O.lm_encode(P(model), sig, P(blk), P(sym), P(out), out.size) > 0
    v1 = model.copy()
    v1[4] = 1
    assert O.lm_encode(P(v1), sig, P(blk), P(sym), P(out), out.size) < 0
    off = model.copy()
    off[12 + 2 * (learned.P_W2 + 64)] ^= 1     # 19/64 -> a neighbour off the grid
    assert O.lm_encode(P(off), sig, P(blk), P(sym), P(out), out.size) < 0


def test_slice_block_enumeration_matches_layout():
    """Blocks cover every node of a section exactly once, in the slice's order."""
    from pentago_b200 import learned
    shape = [45, 19, 72, 8]
    b, n, off = learned.section_blocks(0, shape)
    assert n.sum() == np.prod(shape)
    order = np.argsort(off)
    assert off[order[0]] == 0
    assert np.array_equal(off[order][1:], np.cumsum(n[order])[:-1])
