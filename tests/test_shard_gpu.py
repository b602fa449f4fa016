"""Shards on the GPU: the permutation and board kernels against the oracle,
and the GPU sharder on the reference's solved database (slices 0..5, 32
shards): every group of every shard file equals the format-2 stream of the
oracle's symbols for that shard (so the files equal the reference
sharder's), shard 7 holds the server-verified values of the reference's
sharder test, and a shard range made in small batches gives the same files."""
import ctypes
import os

import numpy as np
import pytest

from tests.oracle import P
from tests.test_shard_cpu import GOLDEN, SH, database_slice, oracle_fns, oracle_symbols, server_value

pytestmark = pytest.mark.gpu


def test_permute_and_board_kernels_match_oracle(cuda, O):
    from pentago_b200 import shard
    lib = oracle_fns(O)
    for s in range(19):
        m = shard.shard_mapping_t(s)
        xs = np.random.default_rng(s).integers(0, m.total(), 3000, dtype=np.uint64)
        assert m.forward_linear(xs).tolist() == [lib.or_shard_permute(s, int(x), 0) for x in xs], s
        assert m.inverse(xs).tolist() == [lib.or_shard_permute(s, int(x), 1) for x in xs], s
        assert m.board(xs).tolist() == [lib.or_shard_board(s, int(x)) for x in xs], s


@pytest.fixture(scope="module")
def shards_dir(tmp_path_factory, cuda):
    from pentago_b200 import shard
    out = tmp_path_factory.mktemp("shards")
    files = shard.sharder(os.path.join(GOLDEN, "db"), str(out), max_slice=SH["max_slice"],
                          total_shards=SH["total_shards"])
    assert len(files) == SH["total_shards"]
    return out


def test_shard_files_match_oracle(O, shards_dir):
    from pentago_b200 import shard
    data = {s: database_slice(O, s)[0] for s in range(SH["max_slice"] + 1)}
    for k in range(SH["total_shards"]):
        f = shard.shard_file_t(str(shards_dir / shard.shard_filename(SH["total_shards"], k)))
        assert (f.header.max_slice, f.header.shard_id, f.header.total_shards) == (SH["max_slice"], k, SH["total_shards"])
        for s in range(SH["max_slice"] + 1):
            sym = oracle_symbols(O, s, SH["total_shards"], k, data[s])
            buf = np.zeros(2 * len(sym) + 1000, np.uint8)
            n = O.rans_encode(P(sym), len(sym), P(buf), len(buf))
            assert f.read_group(s) == buf[:n].tobytes(), (k, s)


def test_shard_holds_server_values(shards_dir):
    from pentago_b200 import shard
    f = shard.shard_file_t(str(shards_dir / shard.shard_filename(SH["total_shards"], SH["shard_id"])))
    found = {}
    for s in range(SH["max_slice"] + 1):
        boards, values = shard.shard_values(f, s)
        found.update(zip(boards.tolist(), values.tolist()))
    for board, val in SH["server_values"]:
        assert server_value(board, found[board]) == val, board


def test_shard_range_in_batches(shards_dir, tmp_path):
    from pentago_b200 import shard
    timings = {}
    shard.sharder(os.path.join(GOLDEN, "db"), str(tmp_path), max_slice=SH["max_slice"],
                  total_shards=SH["total_shards"], shard_range=(9, 14), memory=300000, chunk_nodes=1000,
                  timings=timings)
    assert timings["batch_shards"] < 5   # several batches, several chunks per slice
    for k in range(9, 14):
        name = shard.shard_filename(SH["total_shards"], k)
        assert (tmp_path / name).read_bytes() == (shards_dir / name).read_bytes(), k
    assert not (tmp_path / shard.shard_filename(SH["total_shards"], 8)).exists()
