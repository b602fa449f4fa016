"""In-core backward sweep over all sections below a root section, on one GPU.

The GPU form of the reference's slice loop (pentago/mpi/toplevel.cc:337-415):
for each slice from 35 down to the root's, compute every block line of every
section into one slice tensor (pg_end_sweep_slice), count wins per section
(pg_section_counts), then free the slice above.  Per-section counts are
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

    Returns {slice: counts-N rows}; with keep_last also the last slice tensor."""
    import torch
    from .slice_store import compressed_slice
    root = int(root)
    if min_slice is None:
        min_slice = sum(sum(c) for c in [[(root >> (16 * q + 8 * k)) & 255 for k in range(2)] for q in range(4)])
    L = capi.lib()
    s_handle = capi.stream_handle(stream)
    child_sigs = np.zeros(0, np.uint64)
    child = None   # the slice above: a raw tensor, or compressed
    results = {}
    top = 35
    if resume is not None:
        from .supertensor import read_slice
        start = _slice_of(resume)
        child_sigs = descendent_sections(root, start)
        _, child_sigs, child = read_slice(resume, child_sigs, stream=stream)
        if compress:
            child = compressed_slice(child, child_sigs, start & 1, stream=stream)
            torch.cuda.empty_cache()
        top = start - 1
    for slice_ in range(top, min_slice - 1, -1):
        sigs = descendent_sections(root, slice_)
        torch.cuda.synchronize()
        off = slice_layout(sigs)
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        if isinstance(child, compressed_slice):
            # every line reads one child section: decompress them one by one
            parent = torch.zeros((int(off[-1]), 8), dtype=torch.int64, device="cuda")
            t0.record()
            for ci, csig in enumerate(child.sigs):
                staging = child.section_nodes(ci, stream)
                capi.check(L.pg_end_sweep_slice_child(capi.ptr(sigs), len(sigs), parent.data_ptr(),
                                                      ctypes.c_uint64(int(csig)), staging.data_ptr(), s_handle))
                del staging
            t1.record()
        else:
            parent = torch.empty((int(off[-1]), 8), dtype=torch.int64, device="cuda")
            t0.record()
            capi.check(L.pg_end_sweep_slice(capi.ptr(sigs), len(sigs), parent.data_ptr(), capi.ptr(child_sigs),
                                            len(child_sigs), child.data_ptr() if child is not None else None,
                                            s_handle))
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
                               "child_nodes": 0 if child is None else
                               int(child.base[-1]) if isinstance(child, compressed_slice) else int(child.shape[0])}
        del child
        torch.cuda.empty_cache()  # the slice above is gone; its HBM must be reusable at 180 GB scale
        if compress and slice_ > min_slice:
            e0 = time.perf_counter()
            child = compressed_slice(parent, sigs, slice_ & 1, stream=stream)
            del parent
            torch.cuda.empty_cache()
            if timings is not None:
                torch.cuda.synchronize()
                timings[slice_].update({"compress_s": time.perf_counter() - e0, "compressed_bytes": child.bytes,
                                        "raw_bytes": child.raw_bytes})
        else:
            child = parent
        child_sigs = sigs
    if keep_last:
        return results, child, child_sigs
    return results


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--root", default="4,4,4,5,4,3,3,3")
    ap.add_argument("--min-slice", type=int, default=None)
    ap.add_argument("--golden", default=None, help="npz of counts_N arrays to compare against")
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
        g = np.load(args.golden)
        ok = True
        for s, rows in res.items():
            gold = {int(r[0]): r for r in g[f"counts_{s}"]}
            ok &= all(np.array_equal(gold[int(r[0])], r) for r in rows)
    total_ms = sum(v["ms"] for v in timings.values())
    nbytes = sum(64 * (v["nodes"] + v["child_nodes"]) for v in timings.values())
    print(json.dumps({"root": args.root, "slices": {str(k): v for k, v in timings.items()}, "kernel_ms": total_ms,
                      "wall_s": wall, "sections": sum(v["sections"] for v in timings.values()),
                      "sections_per_s": sum(v["sections"] for v in timings.values()) / (total_ms / 1e3),
                      "algorithmic_GBps": nbytes / (total_ms / 1e3) / 1e9, "golden_counts_match": ok,
                      "peak_GB": torch.cuda.max_memory_allocated() / 1e9}))


if __name__ == "__main__":
    main()
