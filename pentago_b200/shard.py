"""Shards of solved positions for training data.

Python mirror of pentago/shard/shard.h and the sharder
(pentago/shard/sharder.cc) over the library's pg_shard_* entry points:
shard_mapping_t, shard_locator_t, shard_header_t, serialize_shard /
write_shard / shard_file_t, shard_filename, and sharder(), which turns
.pentago slice files (the reference's solved database, or this library's
own sweep checkpoints) into .pentago.shard files.

The sharder's work runs on the GPU: blocks are read and unfiltered there
(pentago_b200.supertensor), scattered into per-shard symbol buffers
(pg_shard_scatter: the permutation of every entry), and every shard's group
of a slice is coded by the format-2 rANS coder (pg_rans_encode_batch), so the
shard files equal the reference sharder's byte for byte.

    python -m pentago_b200.shard --max-slice 5 --shards 32 DB_DIR OUT_DIR [--range lo:hi]
"""
import ctypes
import os

import numpy as np

from . import capi, rans

SHARD_MAGIC = b"pentago shard      \n"
HEADER_SIZE = 36
VERSION = 2


def _device():
    import torch
    return torch.device("cuda", torch.cuda.current_device())


class shard_mapping_t:
    """(section, position, rotation) <-> shuffled index of one slice (shard.h:42-80)."""

    def __init__(self, slice_):
        L = capi.lib()
        n = capi.check(L.pg_shard_sections(slice_, None, 0))
        sigs = np.zeros(max(n, 1), np.uint64)
        capi.check(L.pg_shard_sections(slice_, capi.ptr(sigs), n))
        self.slice = slice_
        self.sections = sigs[:n]
        self.section_id = {int(s): i for i, s in enumerate(self.sections)}
        self._total = int(capi.check(L.pg_shard_total(slice_)))

    def total(self):
        return self._total

    def _apply(self, x, op):
        import torch
        t = torch.as_tensor(np.ascontiguousarray(x, dtype=np.uint64).view(np.int64)).to(_device())
        out = torch.empty_like(t)
        if op == "board":
            capi.check(capi.lib().pg_shard_boards(self.slice, t.data_ptr(), t.numel(), out.data_ptr(),
                                                  capi.stream_handle()))
        else:
            capi.check(capi.lib().pg_shard_permute(self.slice, t.data_ptr(), t.numel(), int(op == "inverse"),
                                                   out.data_ptr(), capi.stream_handle()))
        return out.cpu().numpy().view(np.uint64)

    def forward_linear(self, linear):
        """Permutation of linear indices (offset[section] + 256 position + rotation)."""
        return self._apply(linear, "forward")

    def inverse(self, shuffled):
        return self._apply(shuffled, "inverse")

    def board(self, shuffled):
        """board_t of shuffled indices (shard.cc:137-168)."""
        return self._apply(shuffled, "board")


class shard_locator_t:
    """Power-of-two round-robin assignment of shuffled indices (shard.h:86-115)."""

    def __init__(self, total_shards, shard_range=None):
        if total_shards <= 0 or total_shards & (total_shards - 1):
            raise ValueError("the shard count must be a power of two")
        self.total_shards = total_shards
        self.shard_mask = total_shards - 1
        self.shard_shift = total_shards.bit_length() - 1
        self.shard_range = shard_range or (0, total_shards)

    def shard(self, shuffled):
        return np.asarray(shuffled, np.uint64) & np.uint64(self.shard_mask)

    def position(self, shuffled):
        return np.asarray(shuffled, np.uint64) >> np.uint64(self.shard_shift)

    def shard_size(self, total, shard):
        return (total + self.shard_mask - shard) >> self.shard_shift

    def shuffled_index(self, shard, position):
        return (np.asarray(position, np.uint64) << np.uint64(self.shard_shift)) | np.uint64(shard)


class shard_header_t:
    """The 36-byte shard file header (shard.h:117-133)."""

    def __init__(self, max_slice=0, shard_id=0, total_shards=0, version=VERSION):
        self.version, self.max_slice, self.shard_id, self.total_shards = version, max_slice, shard_id, total_shards

    def pack(self):
        return SHARD_MAGIC + np.array([self.version, self.max_slice, self.shard_id, self.total_shards], "<u4").tobytes()

    @staticmethod
    def unpack(data):
        """Checks as shard_header_t::unpack (shard.cc:189-209)."""
        if len(data) < HEADER_SIZE or bytes(data[:20]) != SHARD_MAGIC:
            raise ValueError("not a shard file (bad magic)")
        v, m, s, t = (int(x) for x in np.frombuffer(bytes(data[20:36]), "<u4"))
        if v != VERSION or m > 18 or s >= t:
            raise ValueError(f"bad shard header (version {v}, max_slice {m}, shard {s} of {t})")
        return shard_header_t(m, s, t, v)


def serialize_shard(header, groups):
    """Header, group offsets (max_slice + 2 little-endian uint32) and the
    serialized groups (shard.cc:211-236)."""
    n = header.max_slice + 1
    if len(groups) != n:
        raise ValueError(f"a shard of max_slice {header.max_slice} holds {n} groups")
    off = [HEADER_SIZE + 4 * (n + 1)]
    for g in groups:
        off.append(off[-1] + len(g))
    if off[-1] > 0xFFFFFFFF:
        raise ValueError("shard larger than 4 GB")
    return header.pack() + np.array(off, "<u4").tobytes() + b"".join(bytes(g) for g in groups)


def write_shard(path, header, groups):
    with open(path, "wb") as f:
        f.write(serialize_shard(header, groups))


class shard_file_t:
    """A shard file read into memory (shard.cc:246-283)."""

    def __init__(self, path_or_bytes):
        data = path_or_bytes if isinstance(path_or_bytes, (bytes, bytearray)) else open(path_or_bytes, "rb").read()
        self.data = bytes(data)
        self.header = shard_header_t.unpack(self.data)
        n = self.header.max_slice + 1
        if len(self.data) < HEADER_SIZE + 4 * (n + 1):
            raise ValueError("truncated shard file")
        self.group_offsets = np.frombuffer(self.data[HEADER_SIZE:HEADER_SIZE + 4 * (n + 1)], "<u4").astype(np.int64)

    def read_group(self, slice_):
        """The serialized format-2 stream of one slice."""
        if not 0 <= slice_ <= self.header.max_slice:
            raise IndexError(f"slice {slice_} not in this shard")
        a, b = int(self.group_offsets[slice_]), int(self.group_offsets[slice_ + 1])
        if not a < b <= len(self.data):
            raise ValueError("bad shard group offsets")
        return self.data[a:b]


def shard_filename(shards, shard):
    """shard-NNNNN-of-NNNNN.pentago.shard, widths from shards - 1 (shard.cc:285-288)."""
    w = len(str(shards - 1))
    return f"shard-{shard:0{w}d}-of-{shards - 1:0{w}d}.pentago.shard"


def parse_shard_total(path):
    base = os.path.basename(path)
    return int(base[base.index("-of-") + 4:base.index(".", base.index("-of-"))]) + 1


def parse_range(text, total):
    """Python-style lo:hi (either side may be empty)."""
    lo, _, hi = text.partition(":")
    lo = int(lo) if lo else 0
    hi = int(hi) if hi else total
    if not 0 <= lo < hi <= total:
        raise ValueError(f"bad shard range {text} of {total}")
    return lo, hi


def shard_values(f, slice_):
    """Decode one slice of a shard file: (boards, values) of its entries in
    shard order (values: 0 tie, 1 black wins, 2 white wins)."""
    if not isinstance(f, shard_file_t):
        f = shard_file_t(f)
    h = f.header
    mapping = shard_mapping_t(slice_)
    loc = shard_locator_t(h.total_shards)
    n = loc.shard_size(mapping.total(), h.shard_id)
    values = rans.decode([f.read_group(slice_)], [n])[0]
    boards = mapping.board(loc.shuffled_index(h.shard_id, np.arange(n, dtype=np.uint64))) if n else np.zeros(0, np.uint64)
    return boards, values


def sharder(input_dir, output_dir, max_slice=18, total_shards=1 << 17, shard_range=None, threads=0,
            memory=None, chunk_nodes=1 << 24, stream=None, timings=None):
    """Turn slice-{0..max_slice}.pentago in input_dir into shard files in
    output_dir (sharder.cc:119-224).  Shards are made in batches that fit
    `memory` bytes of GPU memory (default: 60% of the free memory); per batch
    and slice every block is read to the GPU (chunk_nodes nodes at a time),
    scattered into the batch's shards and each shard's group is coded there."""
    import time
    import torch
    from . import supertensor
    loc = shard_locator_t(total_shards)
    lo, hi = shard_range or (0, total_shards)
    mappings = [shard_mapping_t(s) for s in range(max_slice + 1)]
    if memory is None:
        memory = int(torch.cuda.mem_get_info()[0] * 0.6) - 64 * chunk_nodes
    # raw symbols of the largest slice plus its coded groups (about half as large)
    per_shard = 2 * loc.shard_size(mappings[max_slice].total(), lo) + 64
    batch = max(1, min(hi - lo, memory // max(per_shard, 1)))
    os.makedirs(output_dir, exist_ok=True)
    dev = _device()
    nodes = torch.empty((chunk_nodes, 8), dtype=torch.int64, device=dev)
    readers = {}
    t_scatter = t_encode = t_read = 0.0
    for b0 in range(lo, hi, batch):
        b1 = min(hi, b0 + batch)
        groups = [[None] * (max_slice + 1) for _ in range(b0, b1)]
        for slice_ in range(max_slice, -1, -1):
            m = mappings[slice_]
            sizes = np.array([loc.shard_size(m.total(), s) for s in range(b0, b1)], np.int64)
            offs = np.zeros(len(sizes) + 1, np.int64)
            offs[1:] = np.cumsum(sizes)
            symbols = torch.zeros(max(int(offs[-1]), 1), dtype=torch.uint8, device=dev)
            if slice_ not in readers:
                readers[slice_] = supertensor.open_supertensors(os.path.join(input_dir, f"slice-{slice_}.pentago"))
            rs = readers[slice_]
            if sorted(int(r.header.section) for r in rs) != sorted(int(s) for s in m.sections):
                raise ValueError(f"slice-{slice_}.pentago does not hold exactly the slice's sections")
            # every block of the slice, chunk by chunk
            items = [(r, b) for r in rs for b in r.header.all_blocks()]
            i = 0
            while i < len(items):
                chunk, used = [], 0
                while i < len(items):
                    r, b = items[i]
                    n = int(np.prod(r.header.block_shape(b)))
                    if chunk and used + n > chunk_nodes:
                        break
                    if n > chunk_nodes:
                        raise ValueError("a block is larger than the chunk")
                    chunk.append((r, b, used))
                    used += n
                    i += 1
                t0 = time.perf_counter()
                for r in {id(r): r for r, _, _ in chunk}.values():
                    mine = [(b, o) for rr, b, o in chunk if rr is r]
                    r.read_blocks([b for b, _ in mine], nodes, [o for _, o in mine], turn=supertensor.RAW,
                                  threads=threads, stream=stream)
                t1 = time.perf_counter()
                blocks = (capi.pg_shard_block_t * len(chunk))()
                for k, (r, b, o) in enumerate(chunk):
                    blocks[k].section = m.section_id[int(r.header.section)]
                    for q in range(4):
                        blocks[k].block[q] = b[q]
                    blocks[k].block_size = r.header.block_size
                    blocks[k].node_offset = o
                # the batch's shards are packed back to back: no offset table needed
                capi.check(capi.lib().pg_shard_scatter(slice_, total_shards, b0, b1, blocks, len(chunk),
                                                       nodes.data_ptr(), supertensor.RAW, symbols.data_ptr(),
                                                       None, capi.stream_handle(stream)))
                torch.cuda.synchronize()
                t_read += t1 - t0
                t_scatter += time.perf_counter() - t1
            t0 = time.perf_counter()
            out, out_off, sz = rans.encode_device(symbols, offs, stream)
            host = out.cpu().numpy()
            for k in range(b1 - b0):
                groups[k][slice_] = host[out_off[k]:out_off[k] + sz[k]].tobytes()
            t_encode += time.perf_counter() - t0
            del symbols, out
        for k, s in enumerate(range(b0, b1)):
            write_shard(os.path.join(output_dir, shard_filename(total_shards, s)),
                        shard_header_t(max_slice, s, total_shards), groups[k])
    if timings is not None:
        timings.update({"read_s": t_read, "scatter_s": t_scatter, "encode_s": t_encode, "batch_shards": batch})
    return [shard_filename(total_shards, s) for s in range(lo, hi)]


def synthetic_slice(slice_, seed=0):
    """Every block (block size 8) of every section of a slice, back to back in
    the end engine's block-major layout, with seeded synthetic on-disk pairs
    (black and white wins disjoint, each bit set with probability 1/4).
    Returns (mapping, pg_shard_block_t array, device nodes)."""
    import torch
    from .end import section_shape
    from .supertensor import section_block_offsets
    m = shard_mapping_t(slice_)
    parts, base = [], 0
    for i, sig in enumerate(m.sections):
        shape = section_shape(int(sig))
        idx, off = section_block_offsets(shape)
        parts.append((i, idx, off + base))
        base += int(np.prod(shape))
    nb = sum(len(p[1]) for p in parts)
    blocks = (capi.pg_shard_block_t * nb)()
    k = 0
    for i, idx, off in parts:
        for b, o in zip(idx, off):
            blocks[k].section = i
            for q in range(4):
                blocks[k].block[q] = int(b[q])
            blocks[k].block_size = 8
            blocks[k].node_offset = int(o)
            k += 1
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    r = lambda: torch.randint(-2**63, 2**63 - 1, (base, 4), dtype=torch.int64, device="cuda", generator=g)
    x, y, z = r(), r(), r()
    nodes = torch.cat([x & y, ~x & z], 1).contiguous()
    del x, y, z
    return m, blocks, nodes


def bench_scatter(slice_=10, total_shards=1024, reps=3):
    """The sharder's GPU work for one slice into every shard of a count:
    scatter (permutation of every entry) and the format-2 coding of each
    shard's group, on a synthetic slice resident in HBM."""
    import torch
    m, blocks, nodes = synthetic_slice(slice_)
    loc = shard_locator_t(total_shards)
    sizes = np.array([loc.shard_size(m.total(), s) for s in range(total_shards)], np.int64)
    offs = np.zeros(total_shards + 1, np.int64)
    offs[1:] = np.cumsum(sizes)
    symbols = torch.empty(int(offs[-1]), dtype=torch.uint8, device="cuda")
    s = capi.stream_handle()
    run = lambda: capi.check(capi.lib().pg_shard_scatter(slice_, total_shards, 0, total_shards, blocks, len(blocks),
                                                         nodes.data_ptr(), 2, symbols.data_ptr(), None, s))
    run()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        run()
    e1.record()
    torch.cuda.synchronize()
    scatter_ms = e0.elapsed_time(e1) / reps
    rans.encode_device(symbols[:1 << 20], np.array([0, 1 << 20], np.int64))  # warm the coder
    torch.cuda.synchronize()
    e0.record()
    out, out_off, sz = rans.encode_device(symbols, offs)
    e1.record()
    torch.cuda.synchronize()
    encode_ms = e0.elapsed_time(e1)
    n = m.total()
    return {"workload": f"slice {slice_} (all {len(m.sections)} sections, {n} entries, synthetic values) "
                        f"into {total_shards} shards", "entries": n, "nodes": int(nodes.shape[0]),
            "blocks": len(blocks), "scatter_ms": scatter_ms, "scatter_entries_per_s": n / (scatter_ms / 1e3),
            "encode_ms": encode_ms, "encode_entries_per_s": n / (encode_ms / 1e3),
            "entries_per_s": n / ((scatter_ms + encode_ms) / 1e3), "coded_bytes": int(sz.sum()),
            "scatter_algorithmic_GBps": (64 * nodes.shape[0] + n) / (scatter_ms / 1e3) / 1e9}


def main():
    import argparse
    import json
    import time
    ap = argparse.ArgumentParser(description="convert .pentago slice files to .pentago.shard files on the GPU")
    ap.add_argument("input_dir", nargs="?")
    ap.add_argument("output_dir", nargs="?")
    ap.add_argument("--bench", type=int, default=None, metavar="SLICE",
                    help="time the scatter and coding of a synthetic slice into all shards instead")
    ap.add_argument("--max-slice", type=int, default=18)
    ap.add_argument("--shards", type=int, default=1024, help="total shard count, a power of two")
    ap.add_argument("--range", default=":")
    ap.add_argument("--threads", type=int, default=0)
    args = ap.parse_args()
    import torch
    capi.check(capi.lib().pg_init())
    torch.zeros(1, device="cuda")
    if args.bench is not None:
        print(json.dumps(bench_scatter(args.bench, args.shards)))
        return
    timings = {}
    t = time.perf_counter()
    files = sharder(args.input_dir, args.output_dir, args.max_slice, args.shards,
                    parse_range(args.range, args.shards), args.threads, timings=timings)
    timings["wall_s"] = time.perf_counter() - t
    timings["files"] = len(files)
    print(json.dumps(timings))


if __name__ == "__main__":
    main()
