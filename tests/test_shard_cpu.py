"""Shards on the CPU: the oracle's shard mapping against the reference's
(compiled in place) on every slice 0..18, its scatter against the
reference's scatter_block on the solved database, and both against the
reference sharder test's server-verified samples; the library's host-side
mapping and the kernels' own permutation and board arithmetic (run on the
host) against the oracle; the shard file format.  No GPU."""
import ctypes
import json
import os

import numpy as np
import pytest

from tests.oracle import P

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
SH = json.load(open(os.path.join(GOLDEN, "shards.json")))


def oracle_fns(O):
    for name in ("or_shard_total", "or_shard_size", "or_shard_permute", "or_shard_board"):
        getattr(O.lib, name).restype = ctypes.c_uint64
    O.lib.or_shard_permute.argtypes = [ctypes.c_int, ctypes.c_uint64, ctypes.c_int]
    O.lib.or_shard_board.argtypes = [ctypes.c_int, ctypes.c_uint64]
    O.lib.or_shard_size.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int]
    O.lib.or_shard_symbols.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                       ctypes.c_void_p]
    return O.lib


def sections(lib, prefix, slice_):
    f = getattr(lib, prefix + "shard_sections")
    n = f(slice_, None, 0)
    out = np.zeros(max(n, 1), np.uint64)
    f(slice_, P(out), n)
    return out[:n]


def count_stones(board):
    n = 0
    for q in range(4):
        v = (int(board) >> (16 * q)) & 0xFFFF
        while v:
            n += v % 3 != 0
            v //= 3
    return n


def server_value(board, v):
    """shard_to_server_value (shard.cc:398-403)."""
    if v == 0:
        return 0
    return 1 if (v == 1) == (count_stones(board) % 2 == 0) else -1


def test_oracle_mapping_matches_reference(O, R):
    lib = oracle_fns(O)
    R.lib.ref_shard_total.restype = ctypes.c_uint64
    for s in range(19):
        a, b = sections(R.lib, "ref_", s), sections(lib, "or_", s)
        assert np.array_equal(a, b), s
        n = lib.or_shard_total(s)
        assert n == R.lib.ref_shard_total(s) == SH["slice_totals"][s]
        xs = np.random.default_rng(s).integers(0, n, 400, dtype=np.uint64)
        for op in (0, 1):
            want = np.zeros_like(xs)
            R.lib.ref_shard_permute(s, P(xs), ctypes.c_int64(len(xs)), op, P(want))
            assert [lib.or_shard_permute(s, int(x), op) for x in xs] == want.tolist(), (s, op)
        want = np.zeros_like(xs)
        R.lib.ref_shard_board(s, P(xs), ctypes.c_int64(len(xs)), P(want))
        assert [lib.or_shard_board(s, int(x)) for x in xs] == want.tolist(), s


def test_library_mapping_matches_oracle(O):
    from pentago_b200 import capi
    lib = oracle_fns(O)
    L = capi.lib()
    for s in range(19):
        assert np.array_equal(sections(L, "pg_", s), sections(lib, "or_", s)), s
        n = L.pg_shard_total(s)
        assert n == lib.or_shard_total(s)
        for shards, shard in ((1, 0), (32, 7), (1 << 17, 12345)):
            assert L.pg_shard_size(s, shards, shard) == lib.or_shard_size(s, shards, shard)
        xs = np.random.default_rng(100 + s).integers(0, n, 500, dtype=np.uint64)
        for op, f in ((0, lambda x: lib.or_shard_permute(s, x, 0)), (1, lambda x: lib.or_shard_permute(s, x, 1)),
                      (2, lambda x: lib.or_shard_board(s, x))):
            got = np.zeros_like(xs)
            capi.check(L.pg_selftest_shard_host(op, s, P(xs), len(xs), P(got)))
            assert got.tolist() == [f(int(x)) for x in xs], (s, op)
    assert L.pg_shard_size(5, 12, 0) == capi.PG_ERR_ARG   # counts are powers of two
    assert L.pg_shard_total(19) == capi.PG_ERR_ARG


@pytest.mark.parametrize("slice_", [0, 1, 2, 3])
def test_permutation_is_a_bijection(slice_):
    from pentago_b200 import capi
    L = capi.lib()
    n = L.pg_shard_total(slice_)
    x = np.arange(n, dtype=np.uint64)
    y, back = np.zeros_like(x), np.zeros_like(x)
    capi.check(L.pg_selftest_shard_host(0, slice_, P(x), n, P(y)))
    capi.check(L.pg_selftest_shard_host(1, slice_, P(y), n, P(back)))
    assert np.array_equal(np.sort(y), x) and np.array_equal(back, x)


def database_slice(O, slice_):
    """The reference's solved slice: {sig: (shape, on-disk pairs row-major)} and its blocks."""
    from pentago_b200 import supertensor
    out, blocks = {}, []
    for r in supertensor.open_supertensors(os.path.join(GOLDEN, "db", f"slice-{slice_}.pentago")):
        h = r.header
        arr = np.zeros(tuple(h.shape) + (8,), np.uint64)
        for b in h.all_blocks():
            raw = np.frombuffer(r.read_block_filtered(b).tobytes(), np.uint64).reshape(-1, 8)
            pair = np.zeros_like(raw)
            O.st_unfilter(P(raw), len(raw), 2, 1, P(pair))
            bs = h.block_shape(b)
            sl = tuple(slice(8 * b[q], 8 * b[q] + bs[q]) for q in range(4))
            arr[sl] = pair.reshape(bs + (8,))
            blocks.append((h.section, b, bs, np.ascontiguousarray(pair)))
        out[h.section] = arr
    return out, blocks


def oracle_symbols(O, slice_, total_shards, shard, data):
    lib = oracle_fns(O)
    secs = sections(lib, "or_", slice_)
    flat = np.ascontiguousarray(np.concatenate([data[int(s)].reshape(-1, 8) for s in secs]))
    base = np.zeros(len(secs), np.int64)
    base[1:] = np.cumsum([np.prod(data[int(s)].shape[:4]) for s in secs])[:-1]
    out = np.zeros(max(lib.or_shard_size(slice_, total_shards, shard), 1), np.uint8)
    lib.or_shard_symbols(slice_, total_shards, shard, P(flat), P(base), P(out))
    return out[:lib.or_shard_size(slice_, total_shards, shard)]


def test_oracle_scatter_matches_reference_on_the_database(O, R):
    for s in range(6):
        data, blocks = database_slice(O, s)
        for shards, shard in ((32, 7), (4, 0)):
            want = oracle_symbols(O, s, shards, shard, data)
            got = np.zeros(max(len(want), 1), np.uint8)
            sigs = np.array([b[0] for b in blocks], np.uint64)
            coords = np.array([b[1] for b in blocks], np.uint8).reshape(-1, 4)
            shapes = np.array([b[2] for b in blocks], np.int32).reshape(-1, 4)
            flat = np.ascontiguousarray(np.concatenate([b[3] for b in blocks]))
            offs = np.zeros(len(blocks), np.int64)
            offs[1:] = np.cumsum([len(b[3]) for b in blocks])[:-1]
            R.lib.ref_shard_scatter(s, shards, shard, len(blocks), P(sigs), P(coords), P(shapes), P(offs), P(flat), P(got))
            assert np.array_equal(got[:len(want)], want), (s, shards, shard)


def test_oracle_shard_matches_server_values(O):
    """Shard 7 of 32 over slices 0..5, decoded by the oracle, holds the
    server-verified values of pentago/shard/sharder_test.cc."""
    lib = oracle_fns(O)
    shards, shard = SH["total_shards"], SH["shard_id"]
    found = {}
    for s in range(SH["max_slice"] + 1):
        data, _ = database_slice(O, s)
        sym = oracle_symbols(O, s, shards, shard, data)
        for i, v in enumerate(sym):
            found[lib.or_shard_board(s, (i << 5) | shard)] = int(v)
    for board, val in SH["server_values"]:
        assert board in found, board
        assert server_value(board, found[board]) == val, board


def test_shard_file_format(O):
    from pentago_b200 import shard
    h = shard.shard_header_t(max_slice=18, shard_id=42, total_shards=100000)
    raw = h.pack()
    assert len(raw) == 36 and raw[:20] == b"pentago shard      \n"
    back = shard.shard_header_t.unpack(raw)
    assert (back.version, back.max_slice, back.shard_id, back.total_shards) == (2, 18, 42, 100000)
    for bad in (b"pentago shart      \n" + raw[20:], raw[:20] + np.array([1, 18, 42, 100000], "<u4").tobytes(),
                raw[:20] + np.array([2, 19, 42, 100000], "<u4").tobytes(), raw[:20] + np.array([2, 5, 7, 7], "<u4").tobytes()):
        with pytest.raises(ValueError):
            shard.shard_header_t.unpack(bad)
    # shard.cc's file round trip: groups of (i * 11 + s * 3) % 3 symbols
    groups = []
    for s in range(6):
        sym = np.array([(i * 11 + s * 3) % 3 for i in range(100 + 37 * s)], np.uint8)
        buf = np.zeros(2 * len(sym) + 1000, np.uint8)
        n = O.rans_encode(P(sym), len(sym), P(buf), len(buf))
        groups.append(buf[:n].tobytes())
    f = shard.shard_file_t(shard.serialize_shard(shard.shard_header_t(5, 5, 13), groups))
    assert (f.header.max_slice, f.header.shard_id, f.header.total_shards) == (5, 5, 13)
    assert [f.read_group(s) for s in range(6)] == groups
    assert shard.shard_filename(32, 7) == "shard-07-of-31.pentago.shard"
    assert shard.shard_filename(1048576, 42) == "shard-0000042-of-1048575.pentago.shard"
    assert shard.parse_shard_total("x/shard-0000042-of-1048575.pentago.shard") == 1048576
