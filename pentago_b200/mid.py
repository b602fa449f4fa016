"""Midsolve: the host-side mirror of the reference's midsolve interface.

``midsolve(raws)`` solves a batch of boards (raw_t = board | middle << 63,
pentago/high/board.h:76) with at least 18 stones on the GPU and returns, per
board, the list of (raw, value) pairs of mid_values_t in the order of
midsolve_traverse (pentago/mid/midengine.cc:127-178).  ``values_device``
keeps them on the device as an (n, 8 + 16*163)-byte buffer in the reference's
wasm layout.
"""
import ctypes

import numpy as np

from . import capi

RECORD_BYTES = capi.MID_VALUES_BYTES


def workspace_size(stones):
    """midsolve_workspace_size (pentago/mid/midengine.cc:44-46)."""
    return capi.check(capi.lib().pg_midsolve_workspace_size(stones))


def scratch_bytes(raws):
    raws = np.ascontiguousarray(raws, dtype=np.uint64)
    out = ctypes.c_int64()
    capi.check(capi.lib().pg_midsolve_scratch_bytes(capi.ptr(raws), len(raws), ctypes.byref(out)))
    return out.value


def values_device(raws, out=None, scratch=None, stream=None):
    """Solve on the device; returns the (n, RECORD_BYTES) uint8 tensor of records."""
    import torch
    raws = np.ascontiguousarray(raws, dtype=np.uint64)
    n = len(raws)
    if out is None:
        out = torch.zeros((n, RECORD_BYTES), dtype=torch.uint8, device="cuda")
    sp = capi.ptr(scratch) if scratch is not None else None
    sb = scratch.numel() * scratch.element_size() if scratch is not None else 0
    capi.check(capi.lib().pg_midsolve_batch(capi.ptr(raws), n, out.data_ptr(), sp, sb, capi.stream_handle(stream)))
    return out


_RECORD = np.dtype([("raw", "<u8"), ("value", "<i4"), ("pad", "<i4")])


def decode(records):
    """Host (n, RECORD_BYTES) uint8 array -> list of [(raw, value), ...] per board."""
    records = np.ascontiguousarray(records, dtype=np.uint8)
    result = []
    for row in records:
        size = int(np.frombuffer(row[:4].tobytes(), np.int32)[0])
        if size < 0:
            raise capi.PentagoError(capi.PG_ERR_BOUNDS, "midsolve workspace bounds check failed")
        ent = np.frombuffer(row[8:8 + 16 * 163].tobytes(), _RECORD)[:size]
        result.append(list(zip(ent["raw"].tolist(), ent["value"].tolist())))
    return result


def selftest_host(raws, supers=False):
    """Run the kernel's own solve single-threaded on the CPU (self-test of the
    kernel arithmetic only).  Returns decoded values (and raw halfsupers)."""
    raws = np.ascontiguousarray(raws, dtype=np.uint64)
    out = np.zeros((len(raws), RECORD_BYTES), np.uint8)
    sup = np.zeros((len(raws), 76), np.uint64) if supers else None
    capi.check(capi.lib().pg_selftest_midsolve_host(capi.ptr(raws), len(raws), capi.ptr(out), capi.ptr(sup)))
    return (decode(out), sup) if supers else decode(out)


def selftest_groups_host(raws, groups):
    """The kernel's solve split into `groups` cooperating host threads (the
    multi-CTA partition of every level).  Returns decoded values."""
    raws = np.ascontiguousarray(raws, dtype=np.uint64)
    out = np.zeros((len(raws), RECORD_BYTES), np.uint8)
    capi.check(capi.lib().pg_selftest_midsolve_groups_host(capi.ptr(raws), len(raws), groups, capi.ptr(out)))
    return decode(out)


def midsolve(raws, stream=None):
    """Solve boards on the GPU and return [(raw, value), ...] per board."""
    out = values_device(raws, stream=stream)
    return decode(out.cpu().numpy())


def random_boards(seed, n, stones, reject_wins=True):
    """Seeded boards with `stones` stones placed uniformly on the 6x6 board
    (black has the extra stone when odd), rejecting boards where either side
    already has five in a row.  Returns raw_t values with middle = 0."""
    from .synthetic import splitmix64
    out = []
    ctr = 0
    while len(out) < n:
        r = splitmix64(seed, 36, ctr)
        ctr += 36
        order = np.argsort(r, kind="stable")
        nb = (stones + 1) // 2
        cells = np.zeros(36, np.int64)
        cells[order[:nb]] = 1
        cells[order[nb:stones]] = 2
        board = board_from_cells(cells)
        if reject_wins and (won(board, 1) or won(board, 2)):
            continue
        out.append(board)
    return np.array(out, dtype=np.uint64)


def board_from_cells(cells):
    """6x6 table (x-major, value 0 empty / 1 black / 2 white) -> board_t
    (from_table, pentago/base/board.cc:83-102)."""
    q = [0] * 4
    for qx in range(2):
        for qy in range(2):
            v = 0
            for i in range(9):
                x, y = i // 3, i % 3
                v += 3 ** i * int(cells[(3 * qx + x) * 6 + 3 * qy + y])
            q[2 * qx + qy] = v
    return q[0] | q[1] << 16 | q[2] << 32 | q[3] << 48


_WIN_PATTERNS = None


def _patterns():
    global _WIN_PATTERNS
    if _WIN_PATTERNS is None:
        pats = []

        def bit(x, y, flip, rot):
            if flip:
                x, y = y, x
            if rot:
                x, y = 5 - y, x
            return 1 << (16 * (2 * (x // 3) + y // 3) + 3 * (x % 3) + y % 3)
        for x in range(2):
            for y in range(2):
                pats.append(sum(bit(2 + x + i, 2 + y + i * (-1 if x == y else 1), 0, 0) for i in range(-2, 3)))
        for flip in (0, 1):
            for x in range(2):
                for y in range(6):
                    pats.append(sum(bit(x + i, y, flip, 0) for i in range(5)))
        for rot in (0, 1):
            for x in range(2):
                pats.append(sum(bit(i + x, i + x, 0, rot) for i in range(5)))
        _WIN_PATTERNS = pats
    return _WIN_PATTERNS


def side_of(board, color):
    s = 0
    for q in range(4):
        quad = (board >> (16 * q)) & 0xFFFF
        for i in range(9):
            if quad % 3 == color:
                s |= 1 << (16 * q + i)
            quad //= 3
    return s


def won(board, color):
    s = side_of(board, color)
    return any(s & p == p for p in _patterns())


def positions(raw):
    """Positions a midsolve of this board evaluates: both passes over every
    level, 128 rotations (one parity) per (s0, s1p) item (mid/midengine.cc:78-107)."""
    from math import comb
    stones = bin(side_of(int(raw) & ((1 << 63) - 1), 1) | side_of(int(raw) & ((1 << 63) - 1), 2)).count("1")
    spots = 36 - stones
    items = sum(comb(spots, n >> 1) * comb(spots - (n >> 1), n - (n >> 1)) for n in range(spots + 1))
    return 2 * 128 * items


def algorithmic_bytes(raw):
    """Bytes a midsolve of this board moves through its workspace: both
    passes, at every level n the (s0, s1p) items (N_n of them) each read
    spots - n child halfsupers and write one, 16 bytes each
    (mid/internal.h:358-408 over the info_t levels, mid/internal.h:37-69)."""
    from math import comb
    b = int(raw) & ((1 << 63) - 1)
    spots = 36 - bin(side_of(b, 1) | side_of(b, 2)).count("1")
    total = 0
    for n in range(spots + 1):
        items = comb(spots, n >> 1) * comb(spots - (n >> 1), n - (n >> 1))
        total += items * (16 * (spots - n) + 16)
    return 2 * total


def bench_boards_26(steps=50, warmup=3, sm_max_mhz=1965.0, trials=5):
    """64 seeded 26-stone boards (13 black, 13 white, no five);
    GPU time per batch from CUDA events (median of `trials` trials), and the
    same batch end to end: boards in from the host through the C ABI and the
    64 result records (mid_values_t) copied back to pinned host memory every
    batch.  Returns the result and the boards."""
    import torch
    raws = random_boards(0, 64, 26)
    pos = sum(positions(r) for r in raws)
    alg = sum(algorithmic_bytes(r) for r in raws)
    out = torch.zeros((len(raws), RECORD_BYTES), dtype=torch.uint8, device="cuda")
    host = torch.empty((len(raws), RECORD_BYTES), dtype=torch.uint8).pin_memory()
    scratch = torch.empty(scratch_bytes(raws), dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()

    def device_batch():
        values_device(raws, out=out, scratch=scratch)

    def e2e_batch():
        values_device(raws, out=out, scratch=scratch)
        host.copy_(out, non_blocking=True)
        stream.synchronize()

    def trial(fn):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(steps):
            fn()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / steps
    for _ in range(warmup):
        device_batch()
        e2e_batch()
    torch.cuda.synchronize()
    # `trials` trials of `steps` batches each; the median trial is reported
    ms = sorted(trial(device_batch) for _ in range(trials))[trials // 2]
    e2e_ms = sorted(trial(e2e_batch) for _ in range(trials))[trials // 2]
    sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    peak = 128 * sms * sm_max_mhz * 1e6 / 1e9
    result = {"workload": "64 seeded 26-stone boards (13 black, 13 white, no five), full midsolve",
              "positions_per_batch": pos, "ms_per_batch": ms, "value": pos / (ms / 1e3),
              "boards_per_s": len(raws) / (ms / 1e3), "unit": "positions/s",
              "roofline": {"bound": "shared memory (each board's workspace lives in its CTA's shared memory)",
                           "achieved": alg / (ms / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                           "frac": alg / (ms / 1e3) / 1e9 / peak,
                           "peak_kind": f"nominal: 128 B per clock per SM x {sms} SMs x {sm_max_mhz:.0f} MHz",
                           "algorithmic_bytes_per_batch": alg,
                           "note": "one CTA per pass of a board: 64 boards occupy 128 SMs"},
              "e2e": {"value": pos / (e2e_ms / 1e3), "unit": "positions/s", "ms_per_batch": e2e_ms,
                      "h2d_bytes_per_step": 8 * len(raws), "d2h_bytes_per_step": RECORD_BYTES * len(raws)}}
    return result, raws
