"""Board values from solved slice files, batched on the GPU.

Python mirror of pentago/data/block_cache.h (reader_block_cache,
block_cache_t) and of value() in pentago/high/check.cc for boards not at a
half move, over pg_lookup_*: boards are located on the GPU, the blocks they
need are read from the .pentago files into a block cache in device memory,
and each board's value is read there.

    cache = reader_block_cache(["slice-4.pentago", "slice-5.pentago"], memory=1 << 30)
    cache.values(boards)   # 1 win, 0 tie, -1 loss for the side to move; MISSING if not in the files
"""
import ctypes
import os

import numpy as np

from . import capi

MISSING = capi.PG_LOOKUP_MISSING


class block_cache_t:
    def __init__(self, paths, memory=1 << 30):
        paths = [os.fsencode(p) for p in paths]
        arr = (ctypes.c_char_p * max(len(paths), 1))(*paths)
        h = ctypes.c_void_p()
        self.handle = None
        capi.check(capi.lib().pg_lookup_open(arr, len(paths), int(memory), ctypes.byref(h)))
        self.handle = h

    def values(self, boards, stream=None):
        """Values of absolute boards (black moves first; the side to move is the
        stone-count parity) for the side to move."""
        b = np.ascontiguousarray(boards, dtype=np.uint64).reshape(-1)
        out = np.zeros(max(len(b), 1), np.int32)
        capi.check(capi.lib().pg_lookup_values(self.handle, capi.ptr(b), len(b), capi.ptr(out),
                                               capi.stream_handle(stream)))
        return out[:len(b)]

    def value(self, board):
        return int(self.values([board])[0])

    def stats(self):
        """(boards served without reading a block, blocks read, cache slots)."""
        out = np.zeros(3, np.int64)
        capi.check(capi.lib().pg_lookup_stats(self.handle, capi.ptr(out)))
        return tuple(int(x) for x in out)

    def close(self):
        if self.handle:
            capi.lib().pg_lookup_close(self.handle)
            self.handle = None

    def __del__(self):
        self.close()


def reader_block_cache(paths, memory=1 << 30):
    """A block cache over slice files (block_cache.cc:85-140)."""
    return block_cache_t(paths, memory)


def bench(paths, nboards=1 << 22, slices=range(6), reps=5, memory=1 << 30):
    """Lookups per second of random positions of the given slices (through
    the shard mapping's boards), with every block already cached, host boards
    in and host values out included."""
    import time
    import torch
    from .shard import shard_mapping_t
    rng = np.random.default_rng(0)
    parts = []
    for s in slices:
        m = shard_mapping_t(s)
        parts.append(m.board(rng.integers(0, m.total(), nboards // len(slices), dtype=np.uint64)))
    boards = np.ascontiguousarray(np.concatenate(parts))
    cache = reader_block_cache(paths, memory)
    t = time.perf_counter()
    cache.values(boards)
    cold = time.perf_counter() - t
    torch.cuda.synchronize()
    t = time.perf_counter()
    for _ in range(reps):
        cache.values(boards)
    warm = (time.perf_counter() - t) / reps
    hits, reads, slots = cache.stats()
    return {"workload": f"{len(boards)} random positions of slices {list(slices)} per call", "boards": len(boards),
            "cold_s": cold, "warm_s": warm, "boards_per_s": len(boards) / warm, "blocks_read": reads,
            "cache_slots": slots}
