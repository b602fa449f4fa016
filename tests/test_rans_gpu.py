"""GPU static rANS: byte-identical to the reference's format v2 (oracle and the
reference engine itself), lossless, and it rejects malformed streams the way
pentago/shard/arithmetic_test.cc:152-221 expects."""
import numpy as np
import pytest

from tests.oracle import P

pytestmark = pytest.mark.gpu


def oracle_encode(C, sym):
    cap = 2 * len(sym) + 1000
    out = np.zeros(cap, np.uint8)
    n = C.rans_encode(P(sym), len(sym), P(out), cap)
    assert n > 0
    return out[:n].tobytes()


def cases():
    rng = np.random.default_rng(9)
    yield np.zeros(0, np.uint8)
    yield np.array([2], np.uint8)
    yield np.array([0, 1, 2, 1, 0, 2, 2], np.uint8)           # fewer symbols than lanes
    yield np.full(1000, 1, np.uint8)                          # constant
    yield rng.integers(0, 3, 12345).astype(np.uint8)          # uniform
    yield np.minimum(rng.geometric(0.7, 100000) - 1, 2).astype(np.uint8)  # skewed
    p = rng.random(300007)
    yield np.where(p < 0.93, 0, np.where(p < 0.99, 1, 2)).astype(np.uint8)


def test_encode_matches_oracle_and_reference_bytes(cuda, O):
    from pentago_b200 import rans
    from tests.oracle import reference
    R = reference()
    syms = list(cases())
    got = rans.encode(syms)
    for s, g in zip(syms, got):
        assert g == oracle_encode(O, s)
        if R is not None:
            assert g == oracle_encode(R, s)


def test_roundtrip_is_lossless(cuda):
    from pentago_b200 import rans
    syms = list(cases())
    back = rans.decode(rans.encode(syms))
    for s, b in zip(syms, back):
        assert np.array_equal(s, b)


def test_decodes_reference_streams(cuda, O):
    from pentago_b200 import rans
    syms = list(cases())
    back = rans.decode([oracle_encode(O, s) for s in syms])
    for s, b in zip(syms, back):
        assert np.array_equal(s, b)


def test_malformed_streams_are_rejected(cuda):
    from pentago_b200 import capi, rans
    good = rans.encode([np.array([0, 1, 2] * 50, np.uint8)])[0]
    bad_version = b"\x03" + good[1:]
    truncated = good[:-3]
    short = good[:20]
    for blob in (bad_version, truncated, short):
        with pytest.raises(capi.PentagoError):
            rans.decode([blob], counts=[150])


def test_node_symbols_convention(cuda):
    """symbol = black wins + 2 white wins for each rotation, from [we-win, we-win-or-tie]."""
    import torch
    from pentago_b200 import rans
    from pentago_b200.synthetic import random_nodes
    nodes = random_nodes(3, 50)
    for turn in (0, 1):
        got = rans.node_symbols(torch.from_numpy(nodes.view(np.int64)).cuda(), turn).cpu().numpy()
        bits = lambda words: np.unpackbits(words.view(np.uint8).reshape(-1, 32), axis=1, bitorder="little")
        win, notlost = bits(nodes[:, :4].copy()), bits(nodes[:, 4:].copy())
        black, white = (win, 1 - notlost) if turn == 0 else (1 - notlost, win)
        assert np.array_equal(got.reshape(50, 256), (black + 2 * white).astype(np.uint8))


def test_gpu_rans_determinism_hashes(cuda):
    import hashlib
    from pentago_b200 import rans
    from tests.test_rans_cpu import DETERMINISM, determinism_symbols
    blobs = rans.encode([determinism_symbols(n).astype(np.uint8) for n, _ in DETERMINISM])
    for (name, want), blob in zip(DETERMINISM, blobs):
        assert hashlib.sha1(blob[60:]).hexdigest() == want, name


def test_gpu_rans_malformed_headers(cuda):
    from pentago_b200 import capi, rans
    from tests.test_rans_cpu import header
    ok = rans.decode([header((10, 10, 10), [0] * 8), header((100, 100, 100), [32] * 8) + bytes(range(256))],
                     counts=[30, 300])
    assert [len(x) for x in ok] == [30, 300] and all((x < 3).all() for x in ok)
    for blob, cnt in ((header((10, 10, 10), [1000] * 8) + bytes(32), 30),
                      (header((2**64 - 1, 2**64 - 1, 1), [0] * 8), 1),
                      (header((1 << 52, 1, 1), [0] * 8), 1)):
        with pytest.raises(capi.PentagoError):
            rans.decode([blob], counts=[cnt])
