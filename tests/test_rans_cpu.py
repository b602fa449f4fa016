"""The oracle's static rANS against the reference's own determinism hashes and
malformed-input cases (pentago/shard/arithmetic_test.cc:108-221).  No GPU."""
import hashlib

import numpy as np
import pytest

from tests.oracle import P

# Determinism vectors of arithmetic_test.cc:108-129: SHA-1 of the concatenated streams
DETERMINISM = [("repeat", "214a767752ee0ed88e361b42abc90ee05a3be0d1"),
               ("zeros", "523749d0496f43a7f8e33bad0c7db2e6edc5b8a6"),
               ("threefry", "b3c12598e8201ef562e982f390ae7e6f4fad91af")]


def threefry2x64(key, ctr):
    """Threefry-2x64-20 (Salmon et al., SC'11), as pentago/utility/threefry.cc uses it."""
    M = (1 << 64) - 1
    rot = [16, 42, 12, 31, 16, 32, 24, 21]
    k0, k1 = key & M, key >> 64 & M
    ks = [k0, k1, 0x1BD11BDAA9FC1A22 ^ k0 ^ k1]
    x0, x1 = (ctr & M) + ks[0] & M, (ctr >> 64 & M) + ks[1] & M
    for r in range(20):
        x0 = x0 + x1 & M
        x1 = ((x1 << rot[r % 8]) | (x1 >> (64 - rot[r % 8]))) & M
        x1 ^= x0
        if r % 4 == 3:
            i = (r + 1) // 4
            x0 = x0 + ks[i % 3] & M
            x1 = x1 + ks[(i + 1) % 3] + i & M
    return x1 << 64 | x0


def determinism_symbols(name):
    if name == "repeat":
        return np.arange(20, dtype=np.int64) % 3
    if name == "zeros":
        return np.zeros(100, np.int64)
    return np.array([threefry2x64(7, i) % 3 for i in range(1000)])


def encode(C, sym):
    sym = np.asarray(sym, np.uint8)
    cap = 2 * len(sym) + 1000
    out = np.zeros(cap, np.uint8)
    n = C.rans_encode(P(sym), len(sym), P(out), cap)
    assert n >= 60
    return out[:n].tobytes()


@pytest.mark.parametrize("name,want", DETERMINISM)
def test_oracle_rans_determinism_hashes(O, name, want):
    blob = encode(O, determinism_symbols(name))
    assert hashlib.sha1(blob[60:]).hexdigest() == want


def test_oracle_rans_matches_reference_and_roundtrips(O, R):
    rng = np.random.default_rng(4)
    for n in (0, 1, 7, 8, 9, 1000, 65537):
        for w in ((1, 1, 1), (70, 20, 10), (1, 0, 0), (0, 0, 1)):
            p = np.array(w, float) / sum(w)
            sym = rng.choice(3, size=n, p=p).astype(np.uint8)
            a, b = encode(O, sym), encode(R, sym)
            assert a == b
            out = np.zeros(max(n, 1), np.uint8)
            assert O.rans_decode(np.frombuffer(a, np.uint8).ctypes.data, len(a), P(out), n) == n
            assert np.array_equal(out[:n], sym)


def header(counts, lens):
    return (np.array([2], "<u4").tobytes() + np.array(counts, "<u8").tobytes() +
            np.array(lens, "<u4").tobytes())


@pytest.mark.parametrize("counts,lens,data,ok", [
    ((10, 10, 10), [0] * 8, b"", True),                 # empty streams decode to valid symbols
    ((0, 0, 0), [0] * 8, b"", True),
    ((100, 100, 100), [32] * 8, bytes(range(256)), True),  # garbage content
    ((10, 10, 10), [1000] * 8, bytes(32), False),       # lengths do not sum to the data
    ((2**64 - 1, 2**64 - 1, 1), [0] * 8, b"", False),    # counts overflow
    ((1 << 52, 1, 1), [0] * 8, b"", False),             # count * 0x3fff overflows
])
def test_oracle_rans_malformed_streams(O, counts, lens, data, ok):
    blob = np.frombuffer(header(counts, lens) + data, np.uint8).copy()
    out = np.zeros(1000, np.uint8)
    n = O.rans_decode(P(blob), len(blob), P(out), 1000)
    if ok:
        assert n == sum(counts) and (out[:n] < 3).all()
    else:
        assert n < 0
