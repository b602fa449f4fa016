"""Slice files (.pentago supertensors) on the CPU: the oracle's filter against
the reference's own interleave; the library's header packing, host-side
block reads and writes against the reference's supertensor test
(pentago/data/supertensor_test.cc: its parameters, block write order and
expected file SHA-1), against the reference's solved database of slices
0..5 (data/slice-N.pentago, whose per-section counts must equal
data/counts-N.npy), and the reader's and writer's error cases.  No GPU."""
import ctypes
import hashlib
import json
import os

import numpy as np
import pytest

from tests.oracle import P

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
ST = json.load(open(os.path.join(GOLDEN, "supertensor.json")))


def threefry_vec(key, ctr):
    """Threefry-2x64-20 of one key over an array of 64-bit counters (the high
    counter word is 0), as utility/threefry.cc computes it; (lo, hi) words."""
    M = np.uint64(0xFFFFFFFFFFFFFFFF)
    rot = [16, 42, 12, 31, 16, 32, 24, 21]
    k0, k1 = np.uint64(key & 0xFFFFFFFFFFFFFFFF), np.uint64(key >> 64)
    ks = [k0, k1, np.uint64(0x1BD11BDAA9FC1A22) ^ k0 ^ k1]
    with np.errstate(over="ignore"):
        x0 = np.asarray(ctr, np.uint64) + ks[0]
        x1 = np.zeros_like(x0) + ks[1]
        for r in range(20):
            x0 = x0 + x1
            x1 = (x1 << np.uint64(rot[r % 8])) | (x1 >> np.uint64(64 - rot[r % 8]))
            x1 ^= x0
            if r % 4 == 3:
                i = (r + 1) // 4
                x0 = x0 + ks[i % 3]
                x1 = x1 + ks[(i + 1) % 3] + np.uint64(i)
    return x0 & M, x1 & M


def random_supers(key, n):
    """random_supers (base/superscore.cc:118-127): n supers, 4 words each."""
    a0, a1 = threefry_vec(key, 2 * np.arange(n, dtype=np.uint64))
    c0, c1 = threefry_vec(key, 2 * np.arange(n, dtype=np.uint64) + np.uint64(1))
    return np.stack([a0, a1, c0, c1], -1)


def test_block_shape():
    from pentago_b200 import supertensor
    st = supertensor.supertensor_header_t(supertensor._plain_header(
        supertensor.section_sig(ST["section"]), supertensor.section_shape(supertensor.section_sig(ST["section"])),
        ST["block_size"], ST["filter"]))
    assert list(st.blocks) == ST["blocks"]


def test_test_data(R):
    """The numpy generator equals the reference's random_supers."""
    got = random_supers(ST["key"], 50)
    want = np.zeros((50, 4), np.uint64)
    R.lib.ref_random_supers(ctypes.c_uint64(0), ctypes.c_uint64(ST["key"]), 50, ctypes.c_void_p(want.ctypes.data))
    assert np.array_equal(got, want)


def reference_blocks():
    """supertensor_test.cc's data: block -> on-disk pairs (n, 8) in its key order."""
    from pentago_b200 import supertensor
    sig = supertensor.section_sig(ST["section"])
    h = supertensor.supertensor_header_t(supertensor._plain_header(sig, supertensor.section_shape(sig),
                                                                    ST["block_size"], ST["filter"]))
    key = ST["key"]
    data = {}
    for b in np.ndindex(*ST["blocks"]):
        n = int(np.prod(h.block_shape(b)))
        data[tuple(b)] = np.ascontiguousarray(random_supers(key, 2 * n).reshape(n, 8))
        key += 1
    return sig, h, data


def test_oracle_filter_matches_reference_interleave(O, R):
    rng = np.random.default_rng(1)
    x = rng.integers(0, 2**63, size=(500, 8), dtype=np.uint64) * np.uint64(2) + rng.integers(0, 2, (500, 8), dtype=np.uint64)
    want = x.copy()
    R.lib.ref_st_interleave(ctypes.c_void_p(want.ctypes.data), ctypes.c_int64(500), 0)
    got = np.zeros_like(x)
    O.st_filter(P(x), 500, 2, 1, P(got))
    assert np.array_equal(got, want)


@pytest.mark.parametrize("turn", [0, 1, 2])
@pytest.mark.parametrize("filt", [0, 1])
def test_oracle_filter_roundtrip_and_conversion(O, turn, filt):
    rng = np.random.default_rng(2)
    win = rng.integers(0, 2**64 - 1, size=(300, 4), dtype=np.uint64, endpoint=True)
    nl = win | rng.integers(0, 2**64 - 1, size=(300, 4), dtype=np.uint64, endpoint=True)
    nodes = np.ascontiguousarray(np.concatenate([win, nl], 1))
    disk = np.zeros_like(nodes)
    O.st_filter(P(nodes), 300, turn, filt, P(disk))
    back = np.zeros_like(nodes)
    O.st_unfilter(P(disk), 300, turn, filt, P(back))
    assert np.array_equal(back, nodes)
    if turn < 2:
        pair = np.zeros_like(nodes)
        O.st_unfilter(P(disk), 300, 2, filt, P(pair))
        black, white = pair[:, :4], pair[:, 4:]
        assert not (black & white).any()  # both sides never win the same rotation
        mover = black if turn == 0 else white
        assert np.array_equal(mover, win)


def test_header_pack_roundtrip():
    from pentago_b200 import capi, supertensor
    sig = supertensor.section_sig([[2, 0], [0, 2], [1, 1], [1, 1]])
    h = supertensor._plain_header(sig, supertensor.section_shape(sig), 6, 1)
    h.valid = 1
    h.index[0], h.index[1], h.index[2] = 864, 301, 12345
    raw = supertensor.pack_header(h)
    assert len(raw) == 85 and raw[:20] == b"pentago supertensor\n"
    assert np.frombuffer(raw[20:24], "<u4")[0] == 3 and raw[24] == 1
    assert np.frombuffer(raw[29:37], np.uint8).tolist() == [2, 0, 0, 2, 1, 1, 1, 1]
    back = supertensor.unpack_header(raw)
    for f, _ in capi.pg_supertensor_header_t._fields_:
        a, b = getattr(h, f), getattr(back, f)
        assert (list(a) == list(b)) if hasattr(a, "__len__") else a == b, f
    with pytest.raises(capi.PentagoError) as e:
        supertensor.unpack_header(b"pentago supertenzor\n" + raw[20:])
    assert e.value.code == capi.PG_ERR_FORMAT


def write_reference_file(path, O, level=None):
    """supertensor_test.cc's file through the host write path (oracle filter)."""
    from pentago_b200 import supertensor
    sig, h, data = reference_blocks()
    w = supertensor.supertensor_writer_t(path, sig, ST["block_size"], ST["filter"], level or ST["level"])
    for b in ST["write_order"]:
        x = data[tuple(b)]
        disk = np.zeros_like(x)
        O.st_filter(P(x), len(x), 2, ST["filter"], P(disk))
        w.write_block_filtered(b, disk.tobytes())
    w.finalize()
    w.close()
    return data


def test_writer_matches_reference_hash_and_reads_back(O, tmp_path):
    from pentago_b200 import supertensor
    path = str(tmp_path / "test.pentago")
    data = write_reference_file(path, O)
    # the expected SHA-1s hold for zlib 1.2.11 and 1.3.x, whose deflate output agrees
    assert hashlib.sha1(open(path, "rb").read()).hexdigest() in ST["sha1"]
    for reader in (supertensor.supertensor_reader_t(path), supertensor.open_supertensors(path)[0]):
        assert reader.header.section == supertensor.section_sig(ST["section"])
        assert reader.header.block_size == ST["block_size"] and reader.header.filter == ST["filter"]
        assert list(reader.header.blocks) == ST["blocks"]
        for b in np.ndindex(*ST["blocks"]):  # another order than the writer's
            raw = np.frombuffer(reader.read_block_filtered(b).tobytes(), np.uint64).reshape(-1, 8)
            pair = np.zeros_like(raw)
            O.st_unfilter(P(raw), len(raw), 2, 1, P(pair))
            assert np.array_equal(pair, data[b])
    assert supertensor.supertensor_slice(path) == 8


def test_xz_blocks_roundtrip(O, tmp_path):
    from pentago_b200 import supertensor
    path = str(tmp_path / "xz.pentago")
    data = write_reference_file(path, O, level=26)
    r = supertensor.supertensor_reader_t(path)
    b = tuple(ST["write_order"][3])
    comp = open(path, "rb").read()
    off = r.blob(b)[2]
    assert comp[off:off + 6] == b"\xfd7zXZ\x00"
    raw = np.frombuffer(r.read_block_filtered(b).tobytes(), np.uint64).reshape(-1, 8)
    pair = np.zeros_like(raw)
    O.st_unfilter(P(raw), len(raw), 2, 1, P(pair))
    assert np.array_equal(pair, data[b])


def test_multiple_section_file(O, tmp_path):
    from pentago_b200 import supertensor
    secs = [[[1, 0], [0, 1], [0, 0], [0, 0]], [[0, 0], [1, 1], [0, 0], [0, 0]]]
    path = str(tmp_path / "multi.pentago")
    ws = supertensor.supertensor_writers(path, secs, block_size=4, filter=1, level=3)
    rng = np.random.default_rng(3)
    data = {}
    for s in (1, 0):   # sections and blocks in any order
        for b in reversed(ws[s].header.all_blocks()):
            n = int(np.prod(ws[s].header.block_shape(b)))
            x = rng.integers(0, 2**63, size=(n, 8), dtype=np.uint64)
            disk = np.zeros_like(x)
            O.st_filter(P(x), n, 2, 1, P(disk))
            ws[s].write_block_filtered(b, disk.tobytes())
            data[s, b] = x
    for w in ws:
        w.finalize()
    del ws
    raw = open(path, "rb").read()
    assert raw[:20] == b"pentago sections   \n"
    readers = supertensor.open_supertensors(path)
    assert [r.header.section for r in readers] == [supertensor.section_sig(c) for c in secs]
    for (s, b), x in data.items():
        got = np.frombuffer(readers[s].read_block_filtered(b).tobytes(), np.uint64).reshape(-1, 8)
        pair = np.zeros_like(got)
        O.st_unfilter(P(got), len(got), 2, 1, P(pair))
        assert np.array_equal(pair, x)


def test_database_counts(O):
    """The reference's solved slices 0..5: every block read by the library,
    unfiltered by the oracle and counted, gives data/counts-N.npy."""
    from pentago_b200 import supertensor
    from pentago_b200.sweep import to_golden
    gold = np.load(os.path.join(GOLDEN, "counts_0_5.npz"))
    for s in range(6):
        readers = supertensor.open_supertensors(os.path.join(GOLDEN, "db", f"slice-{s}.pentago"))
        rows = {int(r[0]): r for r in gold[f"counts_{s}"]}
        assert sorted(r.header.section for r in readers) == sorted(rows)
        for r in readers:
            assert r.header.block_size == 8 and r.header.filter == 1 and r.header.stones == s
            total = np.zeros(3, np.uint64)
            for b in r.header.all_blocks():
                raw = np.frombuffer(r.read_block_filtered(b).tobytes(), np.uint64).reshape(-1, 8)
                nodes = np.zeros_like(raw)
                O.st_unfilter(P(raw), len(raw), s & 1, 1, P(nodes))
                c = np.zeros(3, np.uint64)
                blk = np.array(b, np.uint8)
                O.count_block_wins(r.header.section, P(blk), P(nodes), P(c))
                total += c
            got = to_golden([r.header.section], [total], s)[0]
            assert np.array_equal(got, rows[r.header.section]), (s, r.header)


def test_reader_errors(tmp_path):
    from pentago_b200 import capi, supertensor
    with pytest.raises(capi.PentagoError) as e:
        supertensor.open_supertensors(str(tmp_path / "missing.pentago"))
    assert e.value.code == capi.PG_ERR_IO
    with pytest.raises(capi.PentagoError) as e:
        supertensor.open_supertensors(os.path.join(GOLDEN, "counts_0_5.npz"))
    assert e.value.code == capi.PG_ERR_ARG
    src = open(os.path.join(GOLDEN, "db", "slice-3.pentago"), "rb").read()
    cases = {"magic.pentago": b"pentago sectionz" + src[16:],          # bad magic
             "version.pentago": src[:20] + b"\x04" + src[21:],          # unknown multiple-file version
             "short.pentago": src[:100],                                # truncated: index unreadable
             "invalid.pentago": src[:32 + 24] + b"\x00" + src[32 + 25:]}  # first section not finalized
    for name, data in cases.items():
        p = tmp_path / name
        p.write_bytes(data)
        with pytest.raises(capi.PentagoError) as e:
            supertensor.open_supertensors(str(p))
        assert e.value.code in (capi.PG_ERR_FORMAT, capi.PG_ERR_IO), name
    # a corrupt block decodes with an error, not garbage
    r = supertensor.open_supertensors(os.path.join(GOLDEN, "db", "slice-3.pentago"))[0]
    off, size = r.blob((0, 0, 0, 0))[2], r.blob((0, 0, 0, 0))[1]
    bad = bytearray(src)
    bad[off + size // 2] ^= 0xFF
    p = tmp_path / "corrupt.pentago"
    p.write_bytes(bytes(bad))
    with pytest.raises(capi.PentagoError) as e:
        supertensor.open_supertensors(str(p))[0].read_block_filtered((0, 0, 0, 0))
    assert e.value.code == capi.PG_ERR_FORMAT


def test_writer_errors(O, tmp_path):
    from pentago_b200 import capi, supertensor
    sig = supertensor.section_sig(ST["section"])
    for bs in (5, 0, 28):
        with pytest.raises(capi.PentagoError) as e:
            supertensor.supertensor_writer_t(str(tmp_path / "a.pentago"), sig, bs, 1, 6)
        assert e.value.code == capi.PG_ERR_ARG
    for level in (0, 10, 30):
        with pytest.raises(capi.PentagoError):
            supertensor.supertensor_writer_t(str(tmp_path / "a.pentago"), sig, 6, 1, level)
    with pytest.raises(capi.PentagoError):
        supertensor.supertensor_writer_t(str(tmp_path / "a.txt"), sig, 6, 1, 6)
    path = str(tmp_path / "partial.pentago")
    w = supertensor.supertensor_writer_t(path, sig, 6, 1, 6)
    _, h, data = reference_blocks()
    b = tuple(ST["write_order"][0])
    w.write_block_filtered(b, data[b].tobytes())
    with pytest.raises(capi.PentagoError) as e:   # the same block twice
        w.write_block_filtered(b, data[b].tobytes())
    assert e.value.code == capi.PG_ERR_ARG
    with pytest.raises(capi.PentagoError) as e:   # outside the block grid
        w.write_block_filtered((2, 0, 0, 0), data[b].tobytes())
    assert e.value.code == capi.PG_ERR_ARG
    with pytest.raises(capi.PentagoError) as e:   # incomplete
        w.finalize()
    assert e.value.code == capi.PG_ERR_ARG
    assert os.path.exists(path)
    w.close()
    assert not os.path.exists(path)   # an unfinished file is removed


def test_slice_index_files_match_the_reference():
    """The .pentago.index of each solved slice 0..5 written from the slice
    file equals the reference's index file byte for byte
    (pentago/high/index.cc write_supertensor_index); every block's blob,
    located through the index, gives the offset and compressed size that the
    reader reports; the index layout predicts the size of the reference's
    index files of slices 6..8."""
    import json
    import tempfile
    from pentago_b200 import supertensor as S
    rng = np.random.default_rng(6)
    for s in range(6):
        path = os.path.join(GOLDEN, "db", f"slice-{s}.pentago")
        want = open(path + ".index", "rb").read()
        with tempfile.TemporaryDirectory() as d:
            data = S.write_index(os.path.join(d, "slice.index"), path)
        assert data == want, s
        readers = S.open_supertensors(path)
        for r in [readers[i] for i in rng.choice(len(readers), min(4, len(readers)), replace=False)]:
            for b in r.header.all_blocks():
                off, size = S.index_blob_location(s, r.header.section, b)
                assert size == S.INDEX_BLOB
                uncompressed, compressed, offset = r.blob(b)
                assert S.index_block_location(data[off:off + size]) == (offset, compressed)
                got = S.index_read_block_filtered(path, data, s, r.header.section, b, uncompressed)
                assert np.array_equal(got, r.read_block_filtered(b))
    sizes = json.load(open(os.path.join(GOLDEN, "index_sizes.json")))
    for s, n in sizes.items():
        sigs = S.index_sections(int(s))
        assert S.INDEX_HEAD + S.INDEX_BLOB * sum(S._section_block_counts(sigs)) == n, s
    with pytest.raises(IndexError):
        S.index_blob_location(5, int(S.index_sections(5)[0]), (60, 0, 0, 0))
