"""Midsolve on the GPU against the oracle and the reference's golden vector."""
import json
import os

import numpy as np
import pytest

from tests.oracle import P

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def oracle_values(O, raw):
    r, v = np.zeros(200, np.uint64), np.zeros(200, np.int32)
    n = O.midsolve(int(raw), P(r), P(v))
    return list(zip(r[:n].tolist(), v[:n].tolist()))


@pytest.mark.parametrize("stones", [35, 33, 31, 30, 29, 28, 27, 26])
def test_midsolve_matches_oracle(cuda, O, stones):
    from pentago_b200 import mid
    raws = mid.random_boards(stones, 6, stones)
    raws = np.concatenate([raws, raws | np.uint64(1 << 63)])  # both half-move states
    got = mid.midsolve(raws)
    for raw, g in zip(raws, got):
        assert g == oracle_values(O, raw), f"board {int(raw)}"


def test_midsolve_64_boards_26_stones(cuda, O):
    """64 seeded 26-stone boards (13 black, 13 white, no existing five)."""
    from pentago_b200 import mid
    raws = mid.random_boards(0, 64, 26)
    got = mid.midsolve(raws)
    for raw, g in zip(raws, got):
        assert g == oracle_values(O, raw)


@pytest.mark.parametrize("stones", [25, 24, 23])
def test_midsolve_global_workspace_matches_oracle(cuda, O, stones):
    from pentago_b200 import mid
    raws = mid.random_boards(100 + stones, 2, stones)
    got = mid.midsolve(raws)
    for raw, g in zip(raws, got):
        assert g == oracle_values(O, raw)


def test_midsolve_golden_18_stones(cuda):
    """pentago/mid/benchmark_test.cc: all 163 results of an 18-stone board."""
    from pentago_b200 import mid
    g = json.load(open(os.path.join(GOLD, "midsolve_18.json")))
    got = mid.midsolve(np.array([g["root"]], np.uint64))[0]
    want = {(b | m << 63): v for b, m, v in g["results"]}
    assert len(got) == 163
    assert dict(got) == want


def test_midsolve_workspace_sizes(cuda):
    from pentago_b200 import mid
    w = json.load(open(os.path.join(GOLD, "workspace.json")))
    for i, size in enumerate(w["sizes"]):
        assert mid.workspace_size(w["first_slice"] + i) == size


def test_group_barrier_wait_runs_out_with_a_status(cuda):
    """The barrier between the CTAs of a board waits a bounded time: a CTA left
    alone gives up, marks the fault (which fails the board's record) and the
    kernel ends."""
    import ctypes
    import time
    from pentago_b200 import capi
    fault = ctypes.c_int(0)
    t0 = time.perf_counter()
    capi.check(capi.lib().pg_debug_barrier_timeout(20000, ctypes.byref(fault)))
    assert fault.value == 1
    assert time.perf_counter() - t0 < 10
