"""Board lookups on the GPU over the reference's solved database (slices
0..5): the server-verified values of the reference sharder test, random
positions against the oracle, boards of sections no file holds, the cache
refusing a call with more distinct blocks than slots, and blocks reused
across calls when evicted and read again."""
import os

import numpy as np
import pytest

from tests.test_lookup_cpu import GOLDEN, SH, database_boards, oracle_values

pytestmark = pytest.mark.gpu

DB = [os.path.join(GOLDEN, "db", f"slice-{s}.pentago") for s in range(6)]


def test_server_values(cuda):
    from pentago_b200 import lookup
    cache = lookup.reader_block_cache(DB, memory=64 << 20)
    boards = [b for b, _ in SH["server_values"]]
    assert cache.values(boards).tolist() == [v for _, v in SH["server_values"]]


def test_random_positions_match_oracle(cuda, O):
    from pentago_b200 import lookup
    boards = database_boards(O, 400, 7)
    want = oracle_values(O, boards)
    cache = lookup.reader_block_cache(DB, memory=1 << 30)
    assert np.array_equal(cache.values(boards), want)
    # a small cache: more distinct blocks than slots in one call is refused,
    # and batches that fit evict and reread blocks with the same results
    from pentago_b200 import capi
    small = lookup.reader_block_cache(DB, memory=8 * 256 * 1024)
    with pytest.raises(capi.PentagoError) as e:
        small.values(boards)
    assert e.value.code == capi.PG_ERR_CAPACITY
    got = np.concatenate([small.values(boards[i:i + 4]) for i in range(0, len(boards), 4)])
    assert np.array_equal(got, want)
    assert np.array_equal(np.concatenate([small.values(boards[i:i + 4]) for i in range(0, len(boards), 4)]), want)


def test_missing_sections(cuda, O):
    from pentago_b200 import lookup
    boards = database_boards(O, 50, 3)
    cache = lookup.reader_block_cache(DB[:3], memory=64 << 20)   # slices 0..2 only
    got = cache.values(boards)
    want = oracle_values(O, boards)
    from tests.test_shard_cpu import count_stones
    low = np.array([count_stones(b) <= 2 for b in boards])
    assert np.array_equal(got[low], want[low])
    assert (got[~low] == lookup.MISSING).all()
