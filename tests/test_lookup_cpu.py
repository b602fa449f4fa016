"""Board lookups on the CPU: the oracle's location of a board in the solved
database (block_cache_t::lookup) gives the reference sharder test's
server-verified values from the real database, and the library's location
arithmetic (the kernel's own code, run on the host) equals the oracle's.
No GPU."""
import ctypes
import os

import numpy as np

from tests.oracle import P
from tests.test_shard_cpu import GOLDEN, SH, oracle_fns


def oracle_locate(O, boards):
    n = len(boards)
    secs, idx, syms, turns = np.zeros(n, np.uint64), np.zeros((n, 4), np.int32), np.zeros(n, np.uint16), np.zeros(n, np.int32)
    for i, b in enumerate(boards):
        s, x, y, t = np.zeros(1, np.uint64), np.zeros(4, np.int32), np.zeros(1, np.uint16), np.zeros(1, np.int32)
        O.lookup_locate(int(b), P(s), P(x), P(y), P(t))
        secs[i], idx[i], syms[i], turns[i] = s[0], x, y[0], t[0]
    return secs, idx, syms, turns


def oracle_values(O, boards):
    """value() of each board from the database fixtures, by the oracle."""
    from pentago_b200 import supertensor
    readers = {}
    for s in range(6):
        for r in supertensor.open_supertensors(os.path.join(GOLDEN, "db", f"slice-{s}.pentago")):
            readers[r.header.section] = r
    secs, idx, syms, turns = oracle_locate(O, boards)
    out = []
    for sec, ix, sym, turn in zip(secs, idx, syms, turns):
        r = readers[int(sec)]
        b = tuple(int(i) // 8 for i in ix)
        bs = r.header.block_shape(b)
        raw = np.frombuffer(r.read_block_filtered(b).tobytes(), np.uint64).reshape(-1, 8)
        pair = np.zeros_like(raw)
        O.st_unfilter(P(raw), len(raw), 2, 1, P(pair))
        I = [int(i) % 8 for i in ix]
        d = pair[((I[0] * bs[1] + I[1]) * bs[2] + I[2]) * bs[3] + I[3]]
        v = -1
        for aggressive in (1, 0):
            sup = (d[4:] if turn else d[:4]) if aggressive else ~(d[:4] if turn else d[4:])
            sup = np.ascontiguousarray(sup, dtype=np.uint64)
            res, sy = np.zeros(4, np.uint64), np.array([sym], np.uint16)
            O.transform_super(P(sy), P(sup), P(res), 1)
            v += int(res[0] & np.uint64(1))
        out.append(v)
    return np.array(out, np.int32)


def database_boards(O, count, seed):
    """Random positions of slices 0..5 (through the shard mapping's boards, all rotations)."""
    lib = oracle_fns(O)
    rng = np.random.default_rng(seed)
    out = []
    for s in range(6):
        n = lib.or_shard_total(s)
        out += [lib.or_shard_board(s, int(x)) for x in rng.integers(0, n, count)]
    return np.array(out, np.uint64)


def test_oracle_lookup_matches_server_values(O):
    boards = [b for b, _ in SH["server_values"]]
    assert oracle_values(O, boards).tolist() == [v for _, v in SH["server_values"]]


def test_library_locate_matches_oracle(O):
    from pentago_b200 import capi
    boards = np.concatenate([np.array([b for b, _ in SH["server_values"]], np.uint64), database_boards(O, 300, 1)])
    n = len(boards)
    secs, idx, syms, turns = np.zeros(n, np.uint64), np.zeros((n, 4), np.int32), np.zeros(n, np.uint16), np.zeros(n, np.int32)
    capi.check(capi.lib().pg_selftest_lookup_locate_host(P(boards), n, P(secs), P(idx), P(syms), P(turns)))
    want = oracle_locate(O, boards)
    for got, w in zip((secs, idx, syms, turns), want):
        assert np.array_equal(got, w)
