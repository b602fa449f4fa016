"""The continuous-batching server: results identical alone and in the mix,
admission under a small scratch budget, and clean close."""
import numpy as np
import pytest

from tests.oracle import P

pytestmark = pytest.mark.gpu


def test_results_same_alone_and_in_mix(cuda):
    """Stone counts 18-30: boards with 12 or more empty spots run as gangs of
    workers sharing the bounded group barrier, beside single-worker boards;
    every result equals the same board solved alone."""
    from pentago_b200 import mid, serve
    raws, stones = serve.request_boards(11, 40, lo=18, hi=30)
    assert (stones <= 21).sum() >= 4, "the mix should hold several gang boards"
    alone = [mid.midsolve(np.array([r], np.uint64))[0] for r in raws]
    arrivals = np.linspace(0, 0.05, len(raws))
    with serve.Server(8 << 30) as S:
        res, lat, wall = serve.run_stream(S, raws, arrivals, timeout=120)
    assert all(r is not None for r in res)
    for a, b in zip(alone, res):
        assert a == b


def test_server_golden_18_stone_board(cuda):
    """The reference's 18-stone benchmark board (pentago/mid/benchmark_test.cc:42-58)
    through the server, alone and among 26-stone boards arriving with it: its
    163 (raw, value) pairs equal the golden ones both times."""
    import json
    import os
    from pentago_b200 import mid, serve
    g = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "midsolve_18.json")))
    want = {(b | m << 63): v for b, m, v in g["results"]}
    others = mid.random_boards(3, 12, 26)
    with serve.Server(8 << 30) as S:
        alone, _, _ = serve.run_stream(S, np.array([g["root"]], np.uint64), np.zeros(1), timeout=120)
        raws = np.concatenate([others[:6], np.array([g["root"]], np.uint64), others[6:]])
        mix, _, _ = serve.run_stream(S, raws, np.linspace(0, 0.01, len(raws)), timeout=120)
    assert len(alone[0]) == 163 and dict(alone[0]) == want
    assert dict(mix[6]) == want
    for r, got in zip(others, mix[:6] + mix[7:]):
        assert got == mid.midsolve(np.array([r], np.uint64))[0]


def test_admission_respects_budget(cuda):
    """A budget that fits only a few 22-stone boards at once refuses the rest
    until results are collected, then serves all of them."""
    import time
    from pentago_b200 import mid, serve
    raws = mid.random_boards(5, 12, 22)
    need = mid.scratch_bytes(raws[:1])
    with serve.Server(3 * need + 4096) as S:
        tickets = []
        for r in raws:
            t = S.submit(r)
            if t is None:
                break
            tickets.append(t)
        assert 1 <= len(tickets) <= 3, "budget should admit at most three boards"
        first = {}
        t0 = time.perf_counter()
        while len(first) < len(tickets) and time.perf_counter() - t0 < 120:
            for t in tickets:
                if t not in first:
                    r = S.poll(t)
                    if r is not None:
                        first[t] = r
        rest, lat, wall = serve.run_stream(S, raws[len(tickets):], np.zeros(len(raws) - len(tickets)), timeout=120)
    res = [first.get(t) for t in tickets] + rest
    assert all(r is not None for r in res)
    for r, got in zip(raws, res):
        assert got == mid.midsolve(np.array([r], np.uint64))[0]


def test_server_matches_oracle_small_boards(cuda, O):
    from pentago_b200 import mid, serve
    from tests.test_mid_gpu import oracle_values
    raws = mid.random_boards(8, 16, 27)
    with serve.Server(1 << 30) as S:
        res, _, _ = serve.run_stream(S, raws, np.zeros(len(raws)), timeout=60)
    for r, got in zip(raws, res):
        assert got == oracle_values(O, r)


def test_idle_workers_leave_and_come_back(cuda, O):
    """The workers' wait for requests is bounded: with nothing submitted they
    leave after about 2 s (the host reads the state), and the next submit
    relaunches them with correct results."""
    import time
    from pentago_b200 import mid, serve
    raws = mid.random_boards(21, 2, 28)
    with serve.Server(1 << 30) as S:
        first, _, _ = serve.run_stream(S, raws[:1], np.zeros(1), timeout=60)
        assert S.state() == 1
        t0 = time.perf_counter()
        while S.state() == 1 and time.perf_counter() - t0 < 30:
            time.sleep(0.2)
        assert S.state() == 2, "idle workers should have left"
        second, _, _ = serve.run_stream(S, raws[1:], np.zeros(1), timeout=60)
        assert S.state() == 1
    for raw, got in zip(raws, first + second):
        r, v = np.zeros(200, np.uint64), np.zeros(200, np.int32)
        n = O.midsolve(int(raw), P(r), P(v))
        assert got == list(zip(r[:n].tolist(), v[:n].tolist()))
