"""pg_midsolve_batch_noalloc: the midsolve entry point for callers that cannot
allocate device memory when they need a solve (for example inside a framework
that owns the whole device memory pool, or a loop that must not wait for an
allocation).  It must give exactly what pg_midsolve_batch gives, call after
call, although every call reuses the same fixed scratch array.

This file is named to be collected last, so a run that stops at its first
failure has already run every other test."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def solve_noalloc(raws):
    import torch
    from pentago_b200 import capi, mid
    raws = np.ascontiguousarray(raws, dtype=np.uint64)
    out = torch.zeros((len(raws), mid.RECORD_BYTES), dtype=torch.uint8, device="cuda")
    capi.check(capi.lib().pg_midsolve_batch_noalloc(capi.ptr(raws), len(raws), out.data_ptr(),
                                                    capi.stream_handle()))
    return mid.decode(out.cpu().numpy())


def solve_allocating(raws):
    from pentago_b200 import mid
    return mid.midsolve(np.ascontiguousarray(raws, dtype=np.uint64))


def test_noalloc_matches_allocating_entry_point_twice_in_a_row(cuda):
    from pentago_b200 import mid
    # first call: shared-memory workspaces (26-30 stones, both half-move states)
    a = np.concatenate([mid.random_boards(71, 6, 26), mid.random_boards(72, 6, 29)])
    a = np.concatenate([a, a | np.uint64(1 << 63)])
    # second call: global workspaces carved from the fixed array (22-24 stones)
    b = np.concatenate([mid.random_boards(73, 1, 22), mid.random_boards(74, 2, 24)])
    got_a = solve_noalloc(a)
    got_b = solve_noalloc(b)
    assert got_a == solve_allocating(a)
    assert got_b == solve_allocating(b)
    # and the first batch again, after the array held the second call's data
    assert solve_noalloc(a) == got_a


def test_noalloc_rejects_boards_beyond_its_scratch(cuda):
    from pentago_b200 import capi, mid
    big = mid.random_boards(75, 2, 20)   # two 20-stone workspaces exceed the fixed array
    with pytest.raises(capi.PentagoError) as e:
        solve_noalloc(big)
    assert e.value.code == capi.PG_ERR_CAPACITY
