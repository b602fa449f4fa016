"""Continuous-batching midsolve server (the C ABI's pg_serve_*), and the
serving benchmark:

    python -m pentago_b200.serve [--requests 600] [--rate 400] [--budget-gb 20]

Requests are seeded boards with stone counts uniform in 18..30 (black to move
when even, white when odd), arriving as a Poisson stream.  It reports p50/p99
latency (arrival to result) and boards/s, next to the same boards solved one
request at a time with pg_midsolve_batch.
"""
import argparse
import ctypes
import json
import time

import numpy as np

from . import capi, mid


class Server:
    def __init__(self, budget_bytes=8 << 30):
        self._h = ctypes.c_void_p()
        capi.check(capi.lib().pg_serve_open(int(budget_bytes), ctypes.byref(self._h)))
        self._rec = capi.pg_mid_values_t()

    def submit(self, raw):
        """Ticket, or None when the ring or the scratch budget is full right now."""
        t = capi.lib().pg_serve_submit(self._h, ctypes.c_uint64(int(raw)))
        if t == capi.PG_ERR_CAPACITY:
            return None
        return capi.check(t)

    def poll(self, ticket):
        """[(raw, value), ...] when solved, else None."""
        r = capi.check(capi.lib().pg_serve_poll(self._h, ticket, ctypes.byref(self._rec)))
        if r == 0:
            return None
        rec = self._rec
        return [(rec.entries[i].raw, rec.entries[i].value) for i in range(rec.size)]

    def state(self):
        """1 running, 2 workers left after idling, 3 closed, 0 never launched."""
        return capi.check(capi.lib().pg_serve_state(self._h))

    def close(self):
        if self._h:
            capi.check(capi.lib().pg_serve_close(self._h))
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def request_boards(seed, n, lo=18, hi=30):
    """n seeded boards with stone counts uniform in [lo, hi]."""
    from .synthetic import splitmix64
    stones = lo + (splitmix64(seed, n) % np.uint64(hi - lo + 1)).astype(np.int64)
    out = []
    for i, s in enumerate(stones):
        out.append(int(mid.random_boards(seed * 1000003 + i, 1, int(s))[0]))
    return np.array(out, np.uint64), stones


def run_stream(server, raws, arrivals, timeout=600.0):
    """Submit raws[i] at time arrivals[i] (seconds from start); returns results
    and latencies."""
    n = len(raws)
    results = [None] * n
    latency = np.zeros(n)
    pending = {}      # ticket -> index
    waiting = []      # indices that arrived but were not admitted yet
    nxt = 0
    t0 = time.perf_counter()
    while (nxt < n or pending or waiting) and time.perf_counter() - t0 < timeout:
        now = time.perf_counter() - t0
        while nxt < n and arrivals[nxt] <= now:
            waiting.append(nxt)
            nxt += 1
        while waiting:
            t = server.submit(raws[waiting[0]])
            if t is None:
                break
            pending[t] = waiting.pop(0)
        for t in list(pending):
            r = server.poll(t)
            if r is not None:
                i = pending.pop(t)
                results[i] = r
                latency[i] = time.perf_counter() - t0 - arrivals[i]
        if not pending and not waiting and nxt < n:
            time.sleep(max(0.0, min(arrivals[nxt] - (time.perf_counter() - t0), 0.001)))
    return results, latency, time.perf_counter() - t0


def one_at_a_time(raws):
    """Baseline: each board alone through pg_midsolve_batch, in sequence, with
    device scratch allocated once up front for the largest board (so no call
    allocates)."""
    import torch
    out = torch.zeros((1, mid.RECORD_BYTES), dtype=torch.uint8, device="cuda")
    need = max(mid.scratch_bytes(np.array([r], np.uint64)) for r in raws)
    scratch = torch.empty(need, dtype=torch.uint8, device="cuda")
    lat = np.zeros(len(raws))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    res = []
    for i, r in enumerate(raws):
        t = time.perf_counter()
        mid.values_device(np.array([r], np.uint64), out=out, scratch=scratch)
        res.append(mid.decode(out.cpu().numpy())[0])
        lat[i] = time.perf_counter() - t
    return res, lat, time.perf_counter() - t0


def queued_latency(arrivals, service):
    """Latencies of a FIFO single server with the given service times under
    the given arrivals (the one-at-a-time baseline under the same stream)."""
    finish, out = 0.0, np.zeros(len(service))
    for i in range(len(service)):
        finish = max(arrivals[i], finish) + service[i]
        out[i] = finish - arrivals[i]
    return out


def bench(requests=400, rate=200.0, trials=3, budget_gb=40.0, seed=4):
    """Config 4: seeded requests with stones uniform in 18..30.  Per trial
    (its own seeded Poisson arrivals): the server under the stream (p50/p99
    latency, arrival to result), the server under overload (every request at
    once: its capacity in boards/s), and the same boards one request at a
    time through pg_midsolve_batch (boards/s, and its latencies under the
    same arrivals as a FIFO queue).  Every result of the stream must equal the
    same board solved alone."""
    import torch
    capi.check(capi.lib().pg_init())
    raws, stones = request_boards(seed, requests)
    budget = int(budget_gb * (1 << 30))
    with Server(budget) as S:  # warm-up
        run_stream(S, raws[:16], np.zeros(16))
    one_at_a_time(raws[:16])
    out = []
    identical = True
    for k in range(trials):
        arrivals = np.cumsum(np.random.default_rng(seed + k).exponential(1.0 / rate, requests))
        with Server(budget) as S:
            res, lat, wall = run_stream(S, raws, arrivals)
        with Server(budget) as S:
            cap_res, _, cap_wall = run_stream(S, raws, np.zeros(requests))
        base_res, base_lat, base_wall = one_at_a_time(raws)
        done = np.array([r is not None for r in res])
        identical &= all(a == b for a, b in zip(res, base_res)) and all(a == b for a, b in zip(cap_res, base_res))
        q = queued_latency(arrivals, base_lat)
        out.append({"p50_ms": float(np.percentile(lat[done], 50) * 1e3),
                    "p99_ms": float(np.percentile(lat[done], 99) * 1e3),
                    "completed": int(done.sum()), "stream_wall_s": wall,
                    "capacity_boards_per_s": requests / cap_wall,
                    "baseline_boards_per_s": requests / base_wall,
                    "baseline_p50_ms_same_arrivals": float(np.percentile(q, 50) * 1e3),
                    "baseline_p99_ms_same_arrivals": float(np.percentile(q, 99) * 1e3)})
    torch.cuda.synchronize()
    med = lambda key: float(np.median([t[key] for t in out]))
    base = [t["baseline_boards_per_s"] for t in out]
    return {"workload": f"{requests} seeded midsolve requests, stones uniform 18..30, Poisson arrivals at "
                        f"{rate:.0f}/s, scratch budget {budget_gb:.0f} GiB; {trials} trials",
            "p50_ms": med("p50_ms"), "p99_ms": med("p99_ms"),
            "capacity_boards_per_s": med("capacity_boards_per_s"),
            "baseline_one_at_a_time_boards_per_s": {"median": float(np.median(base)), "min": min(base),
                                                    "max": max(base)},
            "capacity_over_baseline_max": med("capacity_boards_per_s") / max(base),
            "baseline_p50_ms_same_arrivals": med("baseline_p50_ms_same_arrivals"),
            "baseline_p99_ms_same_arrivals": med("baseline_p99_ms_same_arrivals"),
            "results_identical_alone_and_in_mix": bool(identical), "trials": out}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--requests", type=int, default=600)
    ap.add_argument("--rate", type=float, default=200.0, help="Poisson arrival rate (requests/s)")
    ap.add_argument("--budget-gb", type=float, default=40.0)
    ap.add_argument("--seed", type=int, default=4)
    ap.add_argument("--baseline", type=int, default=200, help="requests for the one-at-a-time baseline")
    args = ap.parse_args()
    import torch
    capi.check(capi.lib().pg_init())
    raws, stones = request_boards(args.seed, args.requests)
    rng = np.random.default_rng(args.seed)
    arrivals = np.cumsum(rng.exponential(1.0 / args.rate, args.requests))
    # warm-up: one board of each size class
    with Server(int(args.budget_gb * (1 << 30))) as S:
        w, _, _ = run_stream(S, raws[:8], np.zeros(8))
        res, lat, wall = run_stream(S, raws, arrivals)
    done = [r is not None for r in res]
    base_res, base_lat, base_wall = one_at_a_time(raws[:args.baseline])
    same = all(a == b for a, b in zip(res[:args.baseline], base_res))
    # The one-at-a-time baseline under the same arrivals: a FIFO queue in front
    # of the measured per-request service times
    finish, queued = 0.0, np.zeros(args.baseline)
    for i in range(args.baseline):
        finish = max(arrivals[i], finish) + base_lat[i]
        queued[i] = finish - arrivals[i]
    print(json.dumps({
        "metric": "midsolve serving latency and throughput", "requests": args.requests,
        "stones": "uniform 18..30", "rate_per_s": args.rate, "completed": int(sum(done)),
        "p50_ms": float(np.percentile(lat[done], 50) * 1e3), "p99_ms": float(np.percentile(lat[done], 99) * 1e3),
        "boards_per_s": float(sum(done) / wall), "wall_s": wall,
        "baseline_one_at_a_time": {"requests": args.baseline, "boards_per_s": float(args.baseline / base_wall),
                                   "service_p50_ms": float(np.percentile(base_lat, 50) * 1e3),
                                   "service_p99_ms": float(np.percentile(base_lat, 99) * 1e3),
                                   "p50_ms_same_arrivals": float(np.percentile(queued, 50) * 1e3),
                                   "p99_ms_same_arrivals": float(np.percentile(queued, 99) * 1e3)},
        "results_identical_alone_and_in_mix": bool(same),
        "p99_by_stones_ms": {int(s): float(np.percentile(lat[(stones == s) & np.array(done)], 99) * 1e3)
                             for s in sorted(set(stones.tolist())) if ((stones == s) & np.array(done)).any()},
    }))


if __name__ == "__main__":
    main()
