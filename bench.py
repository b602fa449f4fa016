"""Benchmark: end-engine block compute on one section, pentago's endgame hot path.

Workload (batched): the 30-stone section [[4,4],[4,4],[4,3],[3,4]]
(shape 160x160x318x318, black to move).  One step computes, for B full 8^4
blocks of that section, the four block lines through each block (one per
quadrant dimension, each the full line, exactly the reference's unit of work
schedule_compute_line), on seeded synthetic child superinfo (win subset of
notlost, ~31% of notlost bits set; pentago_b200/synthetic.py).  Every line
has its own child input and output region, as in the reference (the four
lines of a block lie side by side in one device buffer per direction, so the
end-to-end leg moves a block with one copy each way).  Inputs and outputs
together exceed the 126 MB L2, so no flush is needed between steps.

Metric: positions/s = parent nodes computed x 256 rotations / second.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--blocks B] [--impl reference]

Under torchrun each rank computes its own B blocks (weak scaling; lines are
independent, there is no data-path collective).
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SECTION = [[4, 4], [4, 4], [4, 3], [3, 4]]
METRIC = "end-block positions/s (bit-exact)"
UNIT = "positions/s"
PROFILE = os.path.join(ROOT, "profiles", "end_line_kernel.md")


def block_of(i):
    """The i-th benchmark block: full 8^4 blocks spread over the section."""
    return (i % 20, (7 * i + 3) % 20, (11 * i + 5) % 39, (13 * i + 1) % 39)


def rank_blocks(blocks, rank):
    """The blocks rank `rank` computes: its own `blocks` consecutive benchmark
    blocks, disjoint from every other rank's (weak scaling, no exchange)."""
    return [block_of(rank * blocks + t) for t in range(blocks)]


def combine_parity(parity, world, device):
    """Every rank's parity check folded into rank 0's record: ok only when
    every rank's lines matched (all ranks take part)."""
    if world == 1:
        return parity
    import torch
    import torch.distributed as dist
    ok = torch.tensor([1 if parity["ok"] else 0], dtype=torch.int32, device=device)
    dist.all_reduce(ok, op=dist.ReduceOp.MIN)
    return dict(parity, ok=bool(ok.item()), scope="rank 0's counts; ok is the AND over ranks")


def max_over_ranks(x, world, device):
    """The slowest rank's time (all ranks take part)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def section_sig(counts):
    """section_t::sig() (pentago/base/section.h:35-42) of [[b0,w0],...,[b3,w3]]."""
    return sum(int(counts[q][k]) << (16 * q + 8 * k) for q in range(4) for k in range(2))


def synthetic():
    """The seeded child generator (pentago_b200/synthetic.py), loaded by file
    path so that the reference arm imports nothing of the package."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("_bench_synthetic", os.path.join(ROOT, "pentago_b200", "synthetic.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def line_seed(t, dim):
    """Seed of the children of the line along `dim` through benchmark block t."""
    return 1000003 * t + dim


def plan_lines(blocks, rank):
    """Line descriptors (without buffers) for this rank's blocks."""
    from pentago_b200 import end
    sig = section_sig(SECTION)
    lines = []
    for t, b in enumerate(rank_blocks(blocks, rank)):
        for dim in range(4):
            bb = tuple(b[i] for i in range(4) if i != dim)
            line = end.Line(sig, dim, bb)
            lines.append((line, end.line_info(line), line_seed(rank * blocks + t, dim)))
    return lines


def reference_lines(R, blocks, rank):
    """The same lines as plan_lines, for the reference engine (oracle/_ref):
    (dim, length, block_base, children, output) with line sizes from the
    reference's own line_data_t."""
    import ctypes
    import numpy as np
    syn = synthetic()
    sig = section_sig(SECTION)
    shape = (ctypes.c_int32 * 4)()
    R.lib.ref_section_shape(ctypes.c_uint64(sig), shape)
    work = []
    for t, b in enumerate(rank_blocks(blocks, rank)):
        for dim in range(4):
            bb = (ctypes.c_uint8 * 3)(*[b[i] for i in range(4) if i != dim])
            length = (shape[dim] + 7) // 8
            nin, nout = ctypes.c_int64(), ctypes.c_int64()
            R.line_sizes(sig, dim, length, bb, ctypes.byref(nin), ctypes.byref(nout))
            work.append((dim, length, bb, syn.random_nodes(line_seed(rank * blocks + t, dim), nin.value),
                         np.zeros((nout.value, 8), np.uint64)))
    return work


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""
    FIELDS = "clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown," \
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, device):
        self.device = device
        self.samples = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) == 6:
                self.samples.append(parts)

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            self.proc.wait()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        import statistics
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples for k in range(4) if s[2 + k] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def measured_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        return {}


def measured_hbm_peak():
    p = measured_peaks()
    if "hbm_gbs" in p:
        return float(p["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled(key, cast=float):
    """A figure of the line kernel's committed ncu summary (a line
    `key: value`); None if absent.  These come from an earlier capture, not
    from this run, and the bench line says so."""
    try:
        for line in open(PROFILE):
            if line.startswith(key + ":"):
                return cast(line.split(":", 1)[1].strip())
    except (OSError, ValueError):
        pass
    return None


def profile_source():
    return {"source": "profile", "kernel_version": profiled("kernel_version", str),
            "captured": profiled("captured", str)}


def profiled_limiter():
    """What bounds the line kernel instead of HBM: its issue and integer-ALU
    pipe activity in the committed ncu capture of the kernel."""
    issue, alu = profiled("issue_active_pct"), profiled("alu_pipe_active_pct")
    if issue is None or alu is None:
        return None
    return dict({"kind": "integer ALU issue and latency", "issue_active_pct": issue, "alu_pipe_active_pct": alu,
                 "capture": "ncu --set full of one end_line_kernel launch, small case"}, **profile_source())


def cpu_reference_rate(seconds=12.0, threads=0, passes=None, warmup=0, blocks=16, rank=0):
    """The reference's own CPU engine (oracle/_ref) on the same block lines
    as the GPU arm (the four lines through each of `blocks` benchmark
    blocks, same children), repeated for about `seconds` (or exactly
    `passes` times after `warmup` untimed passes)."""
    from tests.oracle import reference, P
    R = reference()
    if R is None:
        return None
    nthreads = R.lib.ref_threads(threads)
    sig = section_sig(SECTION)
    work = reference_lines(R, blocks, rank)

    def one_pass():
        n = 0
        for dim, length, bb, inp, out in work:
            R.compute_line(sig, dim, length, bb, P(inp), P(out), 0)
            n += out.shape[0]
        return n
    for _ in range(warmup):
        one_pass()
    nodes = done = 0
    t0 = time.perf_counter()
    while True:
        nodes += one_pass()
        done += 1
        el = time.perf_counter() - t0
        if (passes is not None and done >= passes) or (passes is None and el >= seconds):
            break
    R.release_threads()   # its idle workers spin; nothing after this timing should share the host with them
    return {"value": nodes * 256 / el, "unit": UNIT, "cores": nthreads, "kind": "reference", "passes": done,
            "ms_per_pass": 1e3 * el / done,
            "sample": f"the {len(work)} block lines of the GPU step (4 through each of {blocks} blocks of section "
                      f"{SECTION}, same children), {done} passes in {el:.1f} s ({nodes} parent nodes), "
                      f"reference engine oracle/_ref on {nthreads} threads"}


def check_against_reference(lines, blocks, rank, per_dim=None):
    """Bit-exact check of the GPU's outputs for the bench lines (the last
    timed step's) against the reference engine on the same children: every
    line, or the first `per_dim` lines of each dimension."""
    import ctypes
    import hashlib
    import numpy as np
    from tests.oracle import reference, oracle, P
    R = reference()
    checker, C = ("reference", R) if R is not None else ("oracle", oracle())
    sig = section_sig(SECTION)
    syn = synthetic()
    seen = [0, 0, 0, 0]
    bad = []
    checked = 0
    for (line, info, seed) in lines:
        d = line.dimension
        if per_dim is not None and seen[d] >= per_dim:
            continue
        seen[d] += 1
        inp = syn.random_nodes(seed, info.input_nodes)
        want = np.zeros((info.output_nodes, 8), np.uint64)
        C.compute_line(sig, d, line.length, (ctypes.c_uint8 * 3)(*line.block_base), P(inp), P(want), 0)
        got = line.output.cpu().numpy().view(np.uint64)
        checked += 1
        if not np.array_equal(got, want):
            bad.append({"dim": d, "block_base": list(line.block_base),
                        "got_sha1": hashlib.sha1(got.tobytes()).hexdigest()[:16],
                        "want_sha1": hashlib.sha1(want.tobytes()).hexdigest()[:16]})
    C.release_threads()
    return {"ok": not bad, "lines_checked": checked, "checker": checker, "mismatches": bad[:4]}


SWEEP_ROOT = [[4, 4], [4, 5], [4, 3], [3, 3]]


def cpu_midsolve_rate(raws, positions, seconds=8.0):
    """The reference's midsolve (oracle/_ref) on the host cores, one board per thread."""
    import numpy as np
    from concurrent.futures import ThreadPoolExecutor
    from tests.oracle import reference, P
    R = reference()
    if R is None:
        return None
    threads = os.cpu_count() or 1

    def solve(raw):
        rr, vv = np.zeros(200, np.uint64), np.zeros(200, np.int32)
        R.midsolve(int(raw), P(rr), P(vv))
    boards = 0
    t0 = time.perf_counter()
    with ThreadPoolExecutor(threads) as ex:
        while time.perf_counter() - t0 < seconds:
            list(ex.map(solve, raws))
            boards += len(raws)
    el = time.perf_counter() - t0
    return {"value": boards / len(raws) * positions / el, "unit": "positions/s", "boards_per_s": boards / el,
            "cores": threads, "kind": "reference",
            "sample": f"the same {len(raws)} boards, repeated for {el:.1f} s, one board per thread"}


def cpu_static_coder_rate(symbols, offsets, seconds=5.0):
    """The reference's format-2 encoder (oracle/_ref) on the host cores, one block per thread."""
    import numpy as np
    from concurrent.futures import ThreadPoolExecutor
    from tests.oracle import reference, P
    R = reference()
    if R is None:
        return None
    blocks = [np.ascontiguousarray(symbols[offsets[i]:offsets[i + 1]]) for i in range(len(offsets) - 1)]
    threads = os.cpu_count() or 1

    def enc(b):
        out = np.zeros(b.size // 2 + 4096, np.uint8)
        return R.rans_encode(P(b), b.size, P(out), out.size)
    done = 0
    t0 = time.perf_counter()
    with ThreadPoolExecutor(threads) as ex:
        while time.perf_counter() - t0 < seconds:
            list(ex.map(enc, blocks))
            done += sum(b.size for b in blocks)
    el = time.perf_counter() - t0
    return {"encode_Msym_per_s": done / el / 1e6, "cores": threads, "kind": "reference",
            "sample": f"{len(blocks)} blocks' symbols, format-2 encode repeated for {el:.1f} s"}


def cpu_scatter_rate(slice_, total_shards, seconds=8.0):
    """The reference's scatter_block (oracle/_ref) on the host cores into every
    shard, on a sample of the slice's blocks sized to about `seconds`."""
    import ctypes
    import numpy as np
    from tests.oracle import reference, P
    from pentago_b200 import shard as shard_mod
    from pentago_b200.end import section_shape
    from pentago_b200.supertensor import section_block_offsets
    R = reference()
    if R is None:
        return None
    R.lib.ref_shard_scatter_seconds.restype = ctypes.c_double
    m = shard_mod.shard_mapping_t(slice_)
    sigs, coords, shapes = [], [], []
    for sig in m.sections:
        shape = np.array(section_shape(int(sig)))
        idx, _ = section_block_offsets(shape)
        for b in idx:
            sigs.append(int(sig))
            coords.append(b)
            shapes.append(np.minimum(8, shape - 8 * b.astype(np.int64)))
    order = np.random.default_rng(0).permutation(len(sigs))
    threads = os.cpu_count() or 1

    def run(k):
        pick = order[:k]
        sg = np.array([sigs[i] for i in pick], np.uint64)
        cd = np.ascontiguousarray(np.array([coords[i] for i in pick], np.uint8))
        sh = np.ascontiguousarray(np.array([shapes[i] for i in pick], np.int32))
        n = sh.prod(1).astype(np.int64)
        off = np.zeros(k, np.int64)
        off[1:] = np.cumsum(n)[:-1]
        rng = np.random.default_rng(1)
        x, y, z = (rng.integers(0, 2**63, size=(int(n.sum()), 4), dtype=np.uint64) for _ in range(3))
        data = np.ascontiguousarray(np.concatenate([x & y, ~x & z], 1))
        sec = R.lib.ref_shard_scatter_seconds(slice_, total_shards, k, P(sg), P(cd), P(sh), P(off), P(data), threads)
        return sec, int(n.sum()) * 256
    k = min(len(sigs), 4 * threads)
    sec, entries = run(k)
    k = min(len(sigs), max(k, int(k * seconds / max(sec, 1e-3))))
    sec, entries = run(k)
    return {"entries_per_s": entries / sec, "cores": threads, "kind": "reference",
            "sample": f"scatter_block of {k} random blocks of slice {slice_} ({entries} entries) into all "
                      f"{total_shards} shards, {sec:.1f} s; format-2 coding not included"}


def cpu_lookup_rate(paths, seconds=5.0):
    """The oracle's restatement of the reference's block-cache lookup and
    value() (a scalar port, one thread) over the same slice files, held
    decompressed in host memory (so no reads are timed), on random positions."""
    import ctypes
    import numpy as np
    from tests.oracle import oracle, P
    from pentago_b200 import supertensor
    from pentago_b200.sweep import slice_layout
    O = oracle()
    for name in ("or_shard_total", "or_shard_board"):
        getattr(O.lib, name).restype = ctypes.c_uint64
    O.lib.or_shard_board.argtypes = [ctypes.c_int, ctypes.c_uint64]
    readers = {}
    slices = []
    for path in paths:
        for r in supertensor.open_supertensors(path):
            readers[r.header.section] = r
            slices.append(r.header.stones)
    secs = np.array(sorted(readers), np.uint64)
    off = slice_layout(secs)
    data = np.zeros((int(off[-1]), 8), np.uint64)
    for i, sig in enumerate(secs):
        r = readers[int(sig)]
        idx, boff = supertensor.section_block_offsets(r.header.shape)
        for b, o in zip(idx, boff):
            raw = np.frombuffer(r.read_block_filtered(tuple(int(x) for x in b)).tobytes(), np.uint64).reshape(-1, 8)
            pair = np.zeros_like(raw)
            O.st_unfilter(P(raw), len(raw), 2, 1, P(pair))
            data[off[i] + o:off[i] + o + len(pair)] = pair
    rng = np.random.default_rng(0)
    boards = np.array([O.lib.or_shard_board(s, int(x)) for s in sorted(set(slices))
                       for x in rng.integers(0, O.lib.or_shard_total(s), 2000)], np.uint64)
    base = np.ascontiguousarray(off[:-1])
    vals = np.zeros(len(boards), np.int32)
    done = 0
    t0 = time.perf_counter()
    while time.perf_counter() - t0 < seconds:
        O.lookup_values(P(boards), len(boards), P(secs), len(secs), P(base), P(data), P(vals))
        done += len(boards)
    el = time.perf_counter() - t0
    return {"boards_per_s": done / el, "cores": 1, "kind": "port",
            "sample": f"{len(boards)} random positions, lookups repeated for {el:.1f} s, blocks in host memory"}


def sweep_summary(timings, wall_s, peak):
    """The full sweep of SWEEP_ROOT (slices 35 -> 30) from its per-slice timings."""
    ms = sum(v["ms"] for v in timings.values())
    slice_bytes = sum(64 * (v["nodes"] + v["child_nodes"]) for v in timings.values())
    line_bytes = sum(v.get("line_bytes", 0) for v in timings.values())
    sections = sum(v["sections"] for v in timings.values())
    per_slice = {str(k): {"kernel_ms": v["ms"], "sections": v["sections"], "lines_per_dim": v.get("lines"),
                          "microlines_per_dim": v.get("microlines"),
                          "line_GBps": v.get("line_bytes", 0) / (v["ms"] / 1e3) / 1e9}
                 for k, v in sorted(timings.items())}
    return {"workload": f"all sections below root {SWEEP_ROOT}, slices 35 -> 30, in HBM",
            "sections": sections, "nodes": sum(v["nodes"] for v in timings.values()), "kernel_ms": ms,
            "arena_ms": sum(v.get("arena_ms", 0.0) for v in timings.values()),
            "arena_GB": max(v.get("arena_GB", 0.0) for v in timings.values()),
            "wall_s": wall_s, "sections_per_s": sections / (ms / 1e3),
            "algorithmic_GBps": line_bytes / (ms / 1e3) / 1e9,
            "algorithmic_bytes": "per block line: 64 B per child node read + 64 B per parent node written "
                                 "(the bench kernel's measure), summed over every line of the sweep",
            "frac_of_hbm_peak": line_bytes / (ms / 1e3) / 1e9 / peak,
            "slice_GBps": slice_bytes / (ms / 1e3) / 1e9,
            "slice_bytes_note": "every node of every slice read once as a child and written once as a parent",
            "per_slice": per_slice}


def cpu_sweep_estimate(root_counts, timings, seconds_per_slice=1.5):
    """The reference engine's time for the same sweep, estimated on the host
    cores: per slice, the four block lines through the first block of the
    slice's largest section are timed on all threads (parent nodes per second),
    and every section's nodes times its non-full dimensions are charged at
    that rate (the slices do not fit host memory, 141.7 GB at the peak)."""
    import ctypes
    import numpy as np
    from tests.oracle import reference, P
    from pentago_b200 import end, sweep
    from pentago_b200.synthetic import random_nodes
    R = reference()
    if R is None:
        return None
    nthreads = R.lib.ref_threads(0)
    root = end.section_sig(root_counts)
    total_s, per_slice = 0.0, {}
    for slice_ in sorted(timings):
        sigs = [int(x) for x in sweep.descendent_sections(root, slice_)]
        work = 0
        for sig in sigs:
            counts = [[(sig >> (16 * q + 8 * k)) & 255 for k in range(2)] for q in range(4)]
            dims = [d for d in range(4) if sum(counts[d]) < 9]
            work += int(np.prod(end.section_shape(sig))) * len(dims)
        big = max(sigs, key=lambda s: int(np.prod(end.section_shape(s))))
        counts = [[(big >> (16 * q + 8 * k)) & 255 for k in range(2)] for q in range(4)]
        lines = []
        for dim in (d for d in range(4) if sum(counts[d]) < 9):
            line = end.Line(big, dim, (0, 0, 0))
            info = end.line_info(line)
            lines.append((dim, line.length, random_nodes(dim + 1, max(info.input_nodes, 1)),
                          np.zeros((info.output_nodes, 8), np.uint64)))
        nodes = 0
        t0 = time.perf_counter()
        while time.perf_counter() - t0 < seconds_per_slice:
            for dim, length, inp, out in lines:
                R.compute_line(big, dim, length, (ctypes.c_uint8 * 3)(0, 0, 0), P(inp), P(out), 0)
                nodes += out.shape[0]
        rate = nodes / (time.perf_counter() - t0)
        per_slice[str(slice_)] = {"line_nodes": work, "nodes_per_s": rate}
        total_s += work / rate
    R.release_threads()
    return {"estimated_s": total_s, "cores": nthreads, "kind": "reference", "per_slice": per_slice,
            "sample": "per slice, the block lines through the first block of its largest section on "
                      f"{nthreads} threads, {seconds_per_slice} s each, charged for every line of the sweep"}


def run_reference_arm(args, rank, world):
    if rank != 0:
        return
    # One step = one pass of the reference engine over the same block lines
    # as one GPU step (4 lines through each of --blocks blocks).
    r = cpu_reference_rate(passes=max(1, args.steps), warmup=args.warmup, blocks=args.blocks)
    if r is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref was not built"}))
        return
    line = {"metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": r["ms_per_pass"], "higher_is_better": True,
            "impl": "reference", "dtype": "u64 bitsets",
            "data": "synthetic",
            "config": workload_config(args.blocks, world, reference=True),
            "cpu_baseline": r, "e2e": {"value": r["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                                       "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def workload_config(blocks, world, reference=False):
    """The config object both arms print: the workload is the same lines."""
    c = {"workload": f"end-engine block compute: 4 full block lines through each of {blocks} "
                     f"8^4 blocks of the 30-stone section {SECTION} per GPU",
         "blocks_per_gpu": blocks, "lines_per_gpu": 4 * blocks,
         "positions": "parent nodes written by each line x 256 rotations: a parent node lies on the lines of "
                      "its quadrant dimensions and is counted once per line, as the reference computes it "
                      "(schedule_compute_line per line, OR-accumulated)",
         "l2": "inputs+outputs exceed L2; no flush between steps", "parallelism": f"lines sharded, dp{world}"}
    if reference:
        c["host_cpu"] = True
    return c


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--blocks", type=int, default=16)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned-coder measurement")
    ap.add_argument("--no-slice-files", action="store_true", help="skip the slice-file filter and I/O measurement")
    ap.add_argument("--no-sharder", action="store_true", help="skip the sharder measurement")
    ap.add_argument("--no-lookup", action="store_true", help="skip the board lookup measurement")
    ap.add_argument("--no-parity", action="store_true", help="skip the check of the timed outputs")
    ap.add_argument("--no-serving", action="store_true", help="skip the serving measurement")
    ap.add_argument("--no-midsolve", action="store_true", help="skip the midsolve measurement")
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        return run_reference_arm(args, rank, world)

    import numpy as np
    import torch
    import torch.distributed as dist
    from pentago_b200 import capi, end
    from pentago_b200.synthetic import random_nodes

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=dev)
    capi.check(capi.lib().pg_init())
    stream = torch.cuda.current_stream()

    # Buffers: the four lines of one block share one pinned host buffer and
    # one device buffer per direction (the end-to-end leg moves a block with
    # one copy in and one copy out); each line reads and writes its own part.
    lines = plan_lines(args.blocks, rank)
    chunk = 4
    blocks = []   # (host in, device in, host out, device out) per block
    in_bytes = out_bytes = 0
    out_nodes = 0
    alg_bytes = 0
    for c in range(0, len(lines), chunk):
        part = lines[c:c + chunk]
        hi = torch.from_numpy(np.concatenate([random_nodes(seed, info.input_nodes) for _, info, seed in part])
                              .view(np.int64)).pin_memory()
        n_out = sum(info.output_nodes for _, info, _ in part)
        ho = torch.empty((n_out, 8), dtype=torch.int64).pin_memory()
        di = hi.to(dev, non_blocking=True)
        do = torch.empty((n_out, 8), dtype=torch.int64, device=dev)
        a = b = 0
        for line, info, _ in part:
            line.input = di[a:a + info.input_nodes]
            line.output = do[b:b + info.output_nodes]
            a += info.input_nodes
            b += info.output_nodes
            out_nodes += info.output_nodes
            alg_bytes += 64 * (info.input_nodes + info.output_nodes)
        blocks.append((hi, di, ho, do))
        in_bytes += hi.numel() * 8
        out_bytes += ho.numel() * 8
    ls = [l for l, _, _ in lines]
    torch.cuda.synchronize()
    plan = end.Plan(ls)

    def step():
        plan.run(stream)

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def slowest(x):
        return max_over_ranks(x, world, dev)

    # Device-resident timing (value + roofline)
    for _ in range(args.warmup):
        step()
    end.check_errors(stream)
    barrier()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    stops = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    with ClockSampler(local) as clocks:
        barrier()
        t_start = torch.cuda.Event(enable_timing=True)
        t_stop = torch.cuda.Event(enable_timing=True)
        t_start.record(stream)
        for k in range(args.steps):
            starts[k].record(stream)
            step()
            stops[k].record(stream)
        t_stop.record(stream)
        barrier()
    end.check_errors(stream)
    elapsed_ms = slowest(t_start.elapsed_time(t_stop))
    kernel_ms = sum(a.elapsed_time(b) for a, b in zip(starts, stops)) / args.steps
    units_all = out_nodes * 256 * args.steps * world
    value = units_all / (elapsed_ms / 1e3)
    # What the timed steps wrote, checked bit for bit against the reference
    # engine on the same children (outside the timed region)
    parity = None if args.no_parity else check_against_reference(lines, args.blocks, rank,
                                                                   per_dim=None if world == 1 else 1)

    # End-to-end through the public API with host buffers.  The blocks go
    # through a three-stage pipeline: one stream copies every block in, one
    # runs each block's plan (its four lines) as its inputs land, one copies
    # every block's results out, so that both copy directions run back to
    # back and the kernels hide between them.
    chunk_plans = [end.Plan(ls[c:c + chunk]) for c in range(0, len(ls), chunk)]
    h2d, comp, d2h = (torch.cuda.Stream(device=dev) for _ in range(3))

    def e2e_step():
        go = torch.cuda.Event()
        go.record(stream)
        for st in (h2d, comp, d2h):
            st.wait_event(go)
        for (hi, di, ho, do), p in zip(blocks, chunk_plans):
            with torch.cuda.stream(h2d):
                di.copy_(hi, non_blocking=True)
            landed = torch.cuda.Event()
            landed.record(h2d)
            comp.wait_event(landed)
            p.run(comp)
            solved = torch.cuda.Event()
            solved.record(comp)
            d2h.wait_event(solved)
            with torch.cuda.stream(d2h):
                ho.copy_(do, non_blocking=True)
        done = torch.cuda.Event()
        done.record(d2h)
        stream.wait_event(done)
        stream.synchronize()

    def copy_step():
        """The e2e step's copies alone, on the same streams and buffers: the
        PCIe bound of the end-to-end figure."""
        go = torch.cuda.Event()
        go.record(stream)
        for st in (h2d, d2h):
            st.wait_event(go)
        for (hi, di, ho, do) in blocks:
            with torch.cuda.stream(h2d):
                di.copy_(hi, non_blocking=True)
            with torch.cuda.stream(d2h):
                ho.copy_(do, non_blocking=True)
        for st in (h2d, d2h):
            done = torch.cuda.Event()
            done.record(st)
            stream.wait_event(done)
        stream.synchronize()

    def timed(fn, n):
        for _ in range(max(1, args.warmup)):
            fn()
        barrier()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(n):
            fn()
        b.record(stream)
        barrier()
        return slowest(a.elapsed_time(b)) / n

    e2e_steps = max(2, min(20, args.steps // 2))
    e2e_ms = timed(e2e_step, e2e_steps)
    e2e_value = out_nodes * 256 * world / (e2e_ms / 1e3)
    copy_ms = timed(copy_step, e2e_steps)
    copy_only = {"ms_per_step": copy_ms, "h2d_bytes": in_bytes, "d2h_bytes": out_bytes,
                 "GBps_both_directions": (in_bytes + out_bytes) / (copy_ms / 1e3) / 1e9,
                 "e2e_frac_of_copy_bound": copy_ms / e2e_ms}

    peak, peak_kind = measured_hbm_peak()
    achieved = alg_bytes / (kernel_ms / 1e3) / 1e9
    traffic_per_node = profiled("dram_bytes_per_parent_node")
    cpu = None
    midsolve = None
    learned = None
    sweep2 = None
    slice_files = None
    sharder = None
    lookups = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_reference_rate(seconds=12.0)
    if rank == 0 and world == 1 and not args.no_midsolve:
        from pentago_b200 import mid
        midsolve, raws0 = mid.bench_boards_26(sm_max_mhz=measured_peaks().get("sm_max_mhz", 1965.0))
        if not args.no_cpu_baseline:
            midsolve["cpu_baseline"] = cpu_midsolve_rate(raws0, midsolve["positions_per_batch"], seconds=8.0)
    serving = None
    if rank == 0 and world == 1 and not args.no_serving:
        # Config 4: the continuous-batching server on a Poisson stream of
        # 18..30-stone requests, against the same boards one at a time
        from pentago_b200 import serve
        serving = serve.bench()

    if rank == 0 and world == 1 and not args.no_learned:
        # The full sweep of SWEEP_ROOT, its section counts checked against the
        # original solve's (data/counts-30..35.npy), then the learned coder
        # trained on its 30-stone slice and run on every block of that slice
        torch.cuda.empty_cache()
        from pentago_b200 import learned as learned_mod
        timings, counts = {}, {}
        learned, sample = learned_mod.run_slice_coding(max_blocks=0, sample_blocks=64, sweep_timings=timings,
                                                       sweep_counts=counts)
        sweep2 = sweep_summary(timings, learned["sweep_s"], measured_hbm_peak()[0])
        gold = np.load(os.path.join(ROOT, "tests", "golden", "counts_30_35.npz"))
        ok = bool(counts)
        for s, rows in counts.items():
            by_sig = {int(r[0]): r for r in gold[f"counts_{s}"]}
            ok &= all(int(r[0]) in by_sig and np.array_equal(by_sig[int(r[0])], r) for r in rows)
        sweep2["golden_counts_match"] = bool(ok)
        sweep2["golden_sections_checked"] = sum(len(rows) for rows in counts.values())
        sweep2["golden_counts_source"] = "tests/golden/counts_30_35.npz (data/counts-30..35.npy of the original solve)"
        if not args.no_cpu_baseline:
            learned["cpu_static_coder"] = cpu_static_coder_rate(*sample, seconds=5.0)
            sweep2["cpu_baseline"] = cpu_sweep_estimate(SWEEP_ROOT, timings, seconds_per_slice=1.5)
            sweep2["kernel_speedup_vs_cpu_estimate"] = sweep2["cpu_baseline"]["estimated_s"] / (sweep2["kernel_ms"] / 1e3)

    if rank == 0 and world == 1 and not args.no_slice_files:
        # The .pentago slice files: filter kernels alone against the HBM
        # roofline, and a real 2.7 GB slice written and read back end to end
        torch.cuda.empty_cache()
        from pentago_b200 import supertensor
        slice_files = {"filter_kernels": supertensor.bench_filter(), "slice_io": supertensor.bench_slice_io(levels=(1,))}
        for k in ("filter", "unfilter"):
            slice_files["filter_kernels"][k]["frac_of_hbm_peak"] = slice_files["filter_kernels"][k]["GBps"] / peak

    if rank == 0 and world == 1 and not args.no_sharder:
        # Training shards: slice 10 (16 G entries, synthetic values) scattered
        # into 1,024 shards and each shard's group coded, resident in HBM
        torch.cuda.empty_cache()
        from pentago_b200 import shard as shard_mod
        sharder = shard_mod.bench_scatter(10, 1024)
        torch.cuda.empty_cache()
        if not args.no_cpu_baseline:
            sharder["cpu_baseline"] = cpu_scatter_rate(10, 1024, seconds=8.0)

    if rank == 0 and world == 1 and not args.no_lookup:
        # Board values from the reference's solved database (slices 0..5)
        # through the device block cache, every block already cached
        import glob
        from pentago_b200 import lookup as lookup_mod
        db = sorted(glob.glob(os.path.join(ROOT, "tests", "golden", "db", "slice-*.pentago")))
        lookups = lookup_mod.bench(db)
        if not args.no_cpu_baseline:
            lookups["cpu_baseline"] = cpu_lookup_rate(db, seconds=5.0)

    parity_all = parity if parity is None else combine_parity(parity, world, dev)
    if rank == 0:
        result = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": elapsed_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64 bitsets", "data": "synthetic",
            "config": dict(workload_config(args.blocks, world),
                           parent_nodes_per_step_per_gpu=out_nodes, bytes_resident_per_gpu=in_bytes + out_bytes),
            "parity": parity_all,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind,
                         "traffic": (traffic_per_node * out_nodes / 4) if traffic_per_node else None,
                         "traffic_note": "dram read + write per launch (mean of the 4 dims) from an earlier ncu "
                                         "capture at full size, scaled by parent nodes",
                         "traffic_source": profile_source(),
                         "algorithmic_bytes_per_step": alg_bytes,
                         "algorithmic_bytes": "64 B per child node read + 64 B per parent node written, per line",
                         "kernel": "end_line_kernel", "launches_per_step": 4,
                         "kernel_ms_per_step": kernel_ms, "limiter": profiled_limiter()},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": in_bytes, "d2h_bytes_per_step": out_bytes,
                    "ms_per_step": e2e_ms, "copy_only": copy_only},
            "gpu_launches": 4 * args.steps,
            "midsolve_64_boards_26_stones": midsolve,
            "serving": serving,
            "sweep_root_30_stones": sweep2,
            "learned_rans_slice_30": learned,
            "slice_files": slice_files,
            "sharder": sharder,
            "lookups": lookups,
            "clocks": clocks.summary(),
        }
        print(json.dumps(result))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
