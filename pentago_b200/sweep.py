"""In-core backward sweep over all sections below a root section, on one GPU.

The GPU form of the reference's slice loop (pentago/mpi/toplevel.cc:337-415):
for each slice from 35 down to the root's, compute every block line of every
section into one slice tensor (pg_end_sweep_slice) and count wins per section
(pg_section_counts).  The slices take turns in the two halves of one device
arena, so only two adjacent slices are ever held.  Per-section counts are
returned in the format of data/counts-N.npy (mpi/io.cc:573-581):
[sig, black wins, white wins, total] over distinct positions.

    python -m pentago_b200.sweep --root 4,4,4,5,4,3,3,3 [--min-slice 30]
        [--checkpoint DIR] [--resume DIR/slice-N.pentago]

runs the sweep and prints one JSON line of timings and HBM throughput.  With
--checkpoint every solved slice is also written as a .pentago slice file
(the reference's format), and --resume starts from such a file.
"""
import argparse
import ctypes
import json
import os
import time

import numpy as np

from . import capi
from .end import section_sig, section_shape


def descendent_sections(root, slice_):
    """Standardized sections root depends on at `slice_`, sorted by sig."""
    L = capi.lib()
    n = capi.check(L.pg_descendent_sections(ctypes.c_uint64(root), slice_, None, 0))
    out = np.zeros(max(n, 1), np.uint64)
    capi.check(L.pg_descendent_sections(ctypes.c_uint64(root), slice_, capi.ptr(out), n))
    return out[:n]


def slice_layout(sigs):
    sigs = np.ascontiguousarray(sigs, dtype=np.uint64)
    off = np.zeros(len(sigs) + 1, np.int64)
    capi.check(capi.lib().pg_slice_layout(capi.ptr(sigs), len(sigs), capi.ptr(off)))
    return off


def to_golden(sigs, counts, slice_):
    """(we-win, we-win-or-tie, total) per section -> counts-N.npy rows."""
    out = np.zeros((len(sigs), 4), np.uint64)
    for i, s in enumerate(sigs):
        wins, losses = counts[i][0], counts[i][2] - counts[i][1]
        if slice_ & 1:
            wins, losses = losses, wins
        out[i] = [s, wins, losses, counts[i][2]]
    return out


def _slice_of(path):
    from .supertensor import supertensor_slice
    return supertensor_slice(path)


def _child_of(sig, dim):
    """The standardized child section of a section along quadrant dim (the
    mover places a stone there), or None when that quadrant is full."""
    c = [[(int(sig) >> (16 * q + 8 * k)) & 255 for k in range(2)] for q in range(4)]
    if c[dim][0] + c[dim][1] >= 9:
        return None
    c[dim][sum(map(sum, c)) & 1] += 1
    std = ctypes.c_uint64()
    t = ctypes.c_int32()
    capi.check(capi.lib().pg_section_standardize(ctypes.c_uint64(section_sig(c)), ctypes.byref(std), ctypes.byref(t)))
    return int(std.value)


def _compressed_slice_step(root, slice_, sigs, off, child, last, checkpoint, level, stream, t0, t1, timings,
                           cache_fraction=0.0):
    """One slice of a compressed sweep, one parent section at a time: the
    section's lines read the (at most four) child sections it needs, decoded
    from the coded child slice one at a time (cache_fraction of the free
    memory may keep decoded sections for later parents), then the
    section is counted, written to the checkpoint, and coded into the new
    slice before the next one is built.  The last slice stays raw.
    Returns (counts rows, coded slice or None, raw slice or None)."""
    import collections
    import time as _time
    import torch
    from .slice_store import compressed_slice
    L = capi.lib()
    s_handle = capi.stream_handle(stream)
    store = None if last else compressed_slice(None, sigs, slice_ & 1)
    raw = torch.empty((int(off[-1]), 8), dtype=torch.int64, device="cuda") if last else None
    writer = None
    if checkpoint is not None:
        from .supertensor import slice_writer
        writer = slice_writer(os.path.join(checkpoint, f"slice-{slice_}.pentago"), slice_, sigs, level)
    counts = np.zeros((len(sigs), 3), np.uint64)
    cache = collections.OrderedDict()
    budget = int(torch.cuda.mem_get_info()[0] * cache_fraction)
    child_index = {int(s): i for i, s in enumerate(child.sigs)} if child is not None else {}
    decode_s = code_s = 0.0
    t0.record()
    for i, psig in enumerate(sigs):
        n = int(off[i + 1] - off[i])
        pbuf = raw[int(off[i]):int(off[i + 1])] if last else torch.empty((n, 8), dtype=torch.int64, device="cuda")
        one = np.array([psig], np.uint64)
        if child is None:
            capi.check(L.pg_end_sweep_slice(capi.ptr(one), 1, pbuf.data_ptr(), None, 0, None, s_handle))
        else:
            pbuf.zero_()
            for csig in sorted({c for c in (_child_of(psig, d) for d in range(4)) if c is not None}):
                if csig not in cache:
                    ci = child_index[csig]
                    need = 64 * int(child.base[ci + 1] - child.base[ci])
                    # room first: decoded sections this section has used are done
                    while cache and sum(64 * v.shape[0] for v in cache.values()) + need > budget:
                        cache.popitem(last=False)
                    e = _time.perf_counter()
                    cache[csig] = child.section_nodes(ci, stream)
                    decode_s += _time.perf_counter() - e
                cache.move_to_end(csig)
                capi.check(L.pg_end_sweep_slice_child(capi.ptr(one), 1, pbuf.data_ptr(), ctypes.c_uint64(csig),
                                                      cache[csig].data_ptr(), s_handle))
            while cache and sum(64 * v.shape[0] for v in cache.values()) > budget:
                cache.popitem(last=False)
        cnt = torch.zeros((1, 3), dtype=torch.int64, device="cuda")
        capi.check(L.pg_section_counts(capi.ptr(one), 1, pbuf.data_ptr(), cnt.data_ptr(), s_handle))
        counts[i] = cnt.cpu().numpy().view(np.uint64)[0]
        if writer is not None:
            writer.write_section(i, pbuf, stream)
        if store is not None:
            e = _time.perf_counter()
            store.add_section(i, pbuf, stream)
            code_s += _time.perf_counter() - e
        del pbuf
    t1.record()
    if writer is not None:
        writer.finalize()
    del cache
    # Freed buffers go back to the device after every slice: kept in torch's
    # cache they would hold up to 169 GB for the root [[4,4],[4,5],[4,3],[3,3]]
    # (against 97.7 GB in use at the peak), for a sweep 17% faster.
    torch.cuda.empty_cache()
    if timings is not None:
        torch.cuda.synchronize()
        timings[slice_] = {"ms": t0.elapsed_time(t1), "sections": len(sigs), "nodes": int(off[-1]),
                           "child_nodes": int(child.base[-1]) if child is not None else 0,
                           "decode_s": decode_s, "code_s": code_s}
        if store is not None:
            timings[slice_].update({"compressed_bytes": store.bytes, "raw_bytes": store.raw_bytes})
    return to_golden(sigs, counts, slice_), store, raw


def line_work(sigs, child_sigs):
    """The block lines of a slice: per quadrant dimension, the number of lines
    and of their microlines (1-D runs of nodes along the line; the sweep
    kernel's CTAs take 4 or 8 of them), and the slice's
    algorithmic bytes counted per line (every line reads its child line and
    writes its parent line once, 64 bytes per node: over a slice, each
    (section, non-full dimension) pair reads its whole child section and
    writes the whole section)."""
    child_nodes = {}
    if len(child_sigs):
        off = slice_layout(child_sigs)
        child_nodes = {int(c): int(off[i + 1] - off[i]) for i, c in enumerate(child_sigs)}
    lines, micro, nbytes = [0] * 4, [0] * 4, 0
    for sig in sigs:
        shape = section_shape(int(sig))
        n = int(np.prod(shape))
        for d in range(4):
            c = _child_of(sig, d)
            if c is None:
                continue
            blocks = [(shape[i] + 7) // 8 for i in range(4)]
            nl = int(np.prod([blocks[i] for i in range(4) if i != d]))
            lines[d] += nl
            # microlines of a line: its cross-section (8^3 unless a cross block is short)
            per_dim = [np.minimum(8, shape[i] - 8 * np.arange(blocks[i])) for i in range(4) if i != d]
            micro[d] += int(np.multiply.outer(np.multiply.outer(per_dim[0], per_dim[1]), per_dim[2]).sum())
            nbytes += 64 * (n + child_nodes.get(c, 0))
    return {"lines": lines, "microlines": micro, "line_bytes": nbytes}


def _arena_nodes(root, chain):
    """Nodes of the two halves of the sweep arena for the slices `chain`
    (top first): slices take turns between the halves, so each half holds
    the largest slice of its turns."""
    nodes = [int(slice_layout(descendent_sections(root, s))[-1]) for s in chain]
    return max(nodes[0::2] + [1]), max(nodes[1::2] + [1])


def sweep(root, min_slice=None, stream=None, keep_last=False, timings=None, checkpoint=None, resume=None, level=6,
          compress=False):
    """Solve all sections below `root` from slice 35 down to `min_slice`.

    checkpoint: a directory that receives every solved slice as
    slice-N.pentago (the reference's slice file format).  resume: a slice
    file (slice N, holding at least the sections the root needs at N) to
    start from instead of solving slices 35..N again.  compress: keep each
    finished slice in HBM as store-coder streams (slice_store.compressed_slice)
    and decompress one child section at a time while the slice below is
    built, for roots whose two largest adjacent slices do not fit raw.

    Without compress the slices live in a device arena of two halves that
    they take turns in, so a slice never overlaps the one above it and
    nothing is allocated or freed while the slices are solved.  (Fresh device
    memory is cleared by the driver before its first use; with an allocation
    per slice that clearing landed inside the kernels of every slice, at up
    to several times their time.)  Slice sizes rise and then fall along a
    sweep, so the halves together hold what the two largest adjacent slices
    need.  The arena is allocated and zeroed once before the first slice
    (timings of the first slice carry that time as "arena_ms"); at the end the
    half without the last slice is released.

    Returns {slice: counts-N rows}; with keep_last also the last slice tensor
    and its sections (without compress, the tensor is a view of its arena
    half, which stays allocated while the caller holds it)."""
    import torch
    root = int(root)
    if min_slice is None:
        min_slice = sum(sum(c) for c in [[(root >> (16 * q + 8 * k)) & 255 for k in range(2)] for q in range(4)])
    L = capi.lib()
    s_handle = capi.stream_handle(stream)
    child_sigs = np.zeros(0, np.uint64)
    child = None   # the slice above: a raw tensor, or compressed
    results = {}
    top = 35
    start = None
    if resume is not None:
        start = _slice_of(resume)
        top = start - 1
    order = list(range(top, min_slice - 1, -1))
    halves = None
    arena_ms = None
    if not compress:
        chain = ([start] if start is not None else []) + order
        sizes = _arena_nodes(root, chain)
        need = 64 * sum(sizes)
        free = torch.cuda.mem_get_info()[0] + torch.cuda.memory_reserved() - torch.cuda.memory_allocated()
        if need > free:
            raise capi.PentagoError(capi.PG_ERR_CAPACITY, f"the sweep holds two adjacent slices raw, {need / 1e9:.1f} GB, "
                                    f"and the device has {free / 1e9:.1f} GB free; sweep with compress=True")
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        halves = [torch.empty((n, 8), dtype=torch.int64, device="cuda") for n in sizes]
        for h in halves:
            h.zero_()
        e1.record()
        torch.cuda.synchronize()
        arena_ms = e0.elapsed_time(e1)
    k = 0  # slices placed so far: even ones in the first half, odd ones in the second

    def place(n):
        nonlocal k
        view = halves[k % 2][:n]
        k += 1
        return view

    if resume is not None:
        from .supertensor import read_slice
        child_sigs = descendent_sections(root, start)
        if compress:
            from .slice_store import compressed_slice
            _, child_sigs, child = read_slice(resume, child_sigs, stream=stream)
            child = compressed_slice(child, child_sigs, start & 1, stream=stream)
            torch.cuda.empty_cache()
        else:
            _, child_sigs, child = read_slice(resume, child_sigs, stream=stream,
                                              out=place(int(slice_layout(child_sigs)[-1])))
    for slice_ in order:
        sigs = descendent_sections(root, slice_)
        torch.cuda.synchronize()
        off = slice_layout(sigs)
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        if compress:
            results[slice_], child, parent = _compressed_slice_step(
                root, slice_, sigs, off, child, slice_ == min_slice, checkpoint, level, stream, t0, t1, timings)
            child_sigs = sigs
            if parent is not None:
                child = parent
            continue
        parent = place(int(off[-1]))
        t0.record()
        capi.check(L.pg_end_sweep_slice(capi.ptr(sigs), len(sigs), parent.data_ptr(), capi.ptr(child_sigs),
                                        len(child_sigs), child.data_ptr() if child is not None else None, s_handle))
        t1.record()
        counts = torch.zeros((len(sigs), 3), dtype=torch.int64, device="cuda")
        capi.check(L.pg_section_counts(capi.ptr(sigs), len(sigs), parent.data_ptr(), counts.data_ptr(), s_handle))
        c = counts.cpu().numpy().view(np.uint64)
        results[slice_] = to_golden(sigs, c, slice_)
        if checkpoint is not None:
            from .supertensor import write_slice
            write_slice(os.path.join(checkpoint, f"slice-{slice_}.pentago"), slice_, sigs, parent, level=level,
                        stream=stream)
        if timings is not None:
            torch.cuda.synchronize()
            timings[slice_] = {"ms": t0.elapsed_time(t1), "sections": len(sigs), "nodes": int(off[-1]),
                               "child_nodes": int(child.shape[0]) if child is not None else 0}
            timings[slice_].update(line_work(sigs, child_sigs))
            if arena_ms is not None and slice_ == order[0]:
                timings[slice_]["arena_ms"] = arena_ms
                timings[slice_]["arena_GB"] = 64 * sum(h.shape[0] for h in halves) / 1e9
        child, child_sigs = parent, sigs
    if halves is not None:
        # back to the device: the half without the last slice, or both halves
        # when the caller does not keep the last slice
        halves = parent = None
        if not keep_last:
            child = None
        torch.cuda.empty_cache()
    if keep_last:
        return results, child, child_sigs
    return results


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--root", default="4,4,4,5,4,3,3,3")
    ap.add_argument("--min-slice", type=int, default=None)
    ap.add_argument("--golden", nargs="+", default=None, help="npz files of counts_N arrays to compare against")
    ap.add_argument("--checkpoint", default=None, help="directory for slice-N.pentago files of every solved slice")
    ap.add_argument("--resume", default=None, help="slice file to start from")
    ap.add_argument("--level", type=int, default=6, help="compression level of checkpoint files (zlib 1-9, xz 20-29)")
    ap.add_argument("--compress", action="store_true", help="keep finished slices compressed in HBM (deeper roots)")
    args = ap.parse_args()
    c = [int(x) for x in args.root.split(",")]
    root = section_sig([[c[0], c[1]], [c[2], c[3]], [c[4], c[5]], [c[6], c[7]]])
    import torch
    capi.check(capi.lib().pg_init())
    torch.zeros(1, device="cuda")  # torch's own CUDA set-up, outside the timed sweep
    torch.cuda.synchronize()
    timings = {}
    t = time.perf_counter()
    res = sweep(root, args.min_slice, timings=timings, checkpoint=args.checkpoint, resume=args.resume,
                level=args.level, compress=args.compress)
    wall = time.perf_counter() - t
    ok = None
    if args.golden:
        g = {}
        for path in args.golden:
            g.update(dict(np.load(path)))
        ok = True
        for s, rows in res.items():
            gold = {int(r[0]): r for r in g[f"counts_{s}"]}
            ok &= all(np.array_equal(gold[int(r[0])], r) for r in rows)
    total_ms = sum(v["ms"] for v in timings.values())
    nbytes = sum(64 * (v["nodes"] + v["child_nodes"]) for v in timings.values())
    print(json.dumps({"root": args.root, "slices": {str(k): v for k, v in timings.items()}, "kernel_ms": total_ms,
                      "arena_ms": sum(v.get("arena_ms", 0.0) for v in timings.values()),
                      "wall_s": wall, "sections": sum(v["sections"] for v in timings.values()),
                      "sections_per_s": sum(v["sections"] for v in timings.values()) / (total_ms / 1e3),
                      "algorithmic_GBps": nbytes / (total_ms / 1e3) / 1e9, "golden_counts_match": ok,
                      "peak_GB": torch.cuda.max_memory_allocated() / 1e9,
                      "peak_reserved_GB": torch.cuda.max_memory_reserved() / 1e9}))


if __name__ == "__main__":
    main()
