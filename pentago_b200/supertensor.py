"""Slice files in the reference's .pentago supertensor format.

Python mirror of pentago/data/supertensor.h (supertensor_header_t,
supertensor_reader_t, supertensor_writer_t, open_supertensors,
supertensor_writers) over the library's pg_supertensor_* entry points, plus
write_slice / read_slice, which store a whole slice tensor of the sweep (the
role of pentago/mpi/io.cc's write_sections / read_sections) for checkpoints
and interchange with the reference's tools.

Blocks read to or written from the GPU are (un)filtered there; compression
(zlib level 1-9, xz level 20-29) runs on host threads.  Node data on the GPU
is a uint64 tensor of 8 words per node: [black wins, white wins] with
turn=RAW (the on-disk pair, what the reference's reader returns), or the end
engine's [we win, we win or tie] with turn = 0 / 1 (side to move).
"""
import ctypes
import functools
import os
import struct

import numpy as np

from . import capi
from .end import section_sig, section_shape

RAW = 2
HEADER_SIZE = 85


def _counts(sig):
    return [[(int(sig) >> (16 * q + 8 * k)) & 255 for k in range(2)] for q in range(4)]


class supertensor_header_t:
    """A section's header (supertensor.h:84-107)."""

    def __init__(self, h):
        self.version = h.version
        self.valid = bool(h.valid)
        self.stones = h.stones
        self.section = h.section
        self.shape = tuple(h.shape)
        self.block_size = h.block_size
        self.blocks = tuple(h.blocks)
        self.filter = h.filter
        self.index = tuple(h.index)

    def block_shape(self, block):
        """Shape of one block (supertensor.cc:25-32)."""
        b, B, bs = block, self.blocks, self.block_size
        if any(not 0 <= b[i] < B[i] for i in range(4)):
            raise IndexError(f"block {tuple(b)} outside {B}")
        return tuple(bs if b[i] + 1 < B[i] else self.shape[i] - bs * (B[i] - 1) for i in range(4))

    def all_blocks(self):
        """Every block of the section, row-major."""
        return [tuple(int(x) for x in b) for b in np.ndindex(*self.blocks)]

    def __repr__(self):
        return (f"supertensor_header_t(section={_counts(self.section)}, shape={self.shape}, "
                f"block_size={self.block_size}, filter={self.filter}, valid={self.valid})")


def pack_header(h):
    """The 85 packed bytes of a pg_supertensor_header_t."""
    out = np.zeros(HEADER_SIZE, np.uint8)
    capi.check(capi.lib().pg_supertensor_header_pack(ctypes.byref(h), capi.ptr(out)))
    return out.tobytes()


def unpack_header(data):
    buf = np.frombuffer(bytes(data[:HEADER_SIZE]), np.uint8).copy()
    h = capi.pg_supertensor_header_t()
    capi.check(capi.lib().pg_supertensor_header_unpack(capi.ptr(buf), ctypes.byref(h)))
    return h


def _block_list(items):
    """[(section index, block)] -> int32 section array, uint8 block array."""
    secs = np.array([s for s, _ in items], np.int32)
    blocks = np.array([list(b) for _, b in items], np.uint8).reshape(-1, 4)
    return np.ascontiguousarray(secs), np.ascontiguousarray(blocks)


class _File:
    """One open file shared by the readers of its sections."""

    def __init__(self, path):
        self.path = path
        self.handle = None
        h = ctypes.c_void_p()
        self.sections = capi.check(capi.lib().pg_supertensor_open(os.fsencode(path), ctypes.byref(h)))
        self.handle = h

    def header(self, s):
        h = capi.pg_supertensor_header_t()
        capi.check(capi.lib().pg_supertensor_header(self.handle, s, ctypes.byref(h)))
        return h

    def close(self):
        if self.handle:
            capi.lib().pg_supertensor_close(self.handle)
            self.handle = None

    def __del__(self):
        self.close()


class supertensor_reader_t:
    """Reader of one section of a .pentago file (supertensor.h:109-166)."""

    def __init__(self, path, _file=None, _section=0):
        self._file = _file if _file is not None else _File(path)
        self._section = _section
        self.header = supertensor_header_t(self._file.header(_section))

    def blob(self, block):
        """(uncompressed size, compressed size, offset) of a block."""
        out = np.zeros(3, np.uint64)
        b = np.array(block, np.uint8)
        capi.check(capi.lib().pg_supertensor_block_blob(self._file.handle, self._section, capi.ptr(b), capi.ptr(out)))
        return tuple(int(x) for x in out)

    def compressed_size(self, block):
        return self.blob(block)[1]

    def uncompressed_size(self, block):
        return self.blob(block)[0]

    def read_block_filtered(self, block, threads=0):
        """The block's decompressed on-disk bytes (host; filtered as stored)."""
        shape = self.header.block_shape(block)
        out = np.zeros(64 * int(np.prod(shape)), np.uint8)
        secs, blocks = _block_list([(self._section, block)])
        off = np.zeros(1, np.int64)
        capi.check(capi.lib().pg_supertensor_read_blocks_host(self._file.handle, 1, capi.ptr(secs), capi.ptr(blocks),
                                                              capi.ptr(out), capi.ptr(off), threads))
        return out

    def read_block(self, block, turn=RAW, threads=0, stream=None):
        """The block's nodes on the GPU: uint64 tensor of shape block_shape + (8,)."""
        import torch
        shape = self.header.block_shape(block)
        out = torch.empty(tuple(shape) + (8,), dtype=torch.int64, device="cuda")
        self.read_blocks([block], out, [0], turn, threads, stream)
        return out

    def read_blocks(self, blocks, nodes, node_offsets, turn=RAW, threads=0, stream=None):
        """Blocks into a device node tensor: block i at node node_offsets[i]."""
        secs, b = _block_list([(self._section, blk) for blk in blocks])
        off = np.ascontiguousarray(node_offsets, dtype=np.int64)
        capi.check(capi.lib().pg_supertensor_read_blocks(self._file.handle, len(blocks), capi.ptr(secs), capi.ptr(b),
                                                         nodes.data_ptr(), capi.ptr(off), turn, threads,
                                                         capi.stream_handle(stream)))


def open_supertensors(path):
    """Readers of every section of a single- or multiple-section file (supertensor.cc:403-435)."""
    f = _File(path)
    return [supertensor_reader_t(path, f, s) for s in range(f.sections)]


def supertensor_slice(path):
    """Stones of the file's first section (supertensor.cc:466-498)."""
    return _File(path).header(0).stones


class _Writer:
    def __init__(self, path, sigs, multiple, block_size, filter, level):
        self.handle = None
        sig_arr = np.ascontiguousarray(sigs, dtype=np.uint64)
        h = ctypes.c_void_p()
        capi.check(capi.lib().pg_supertensor_create(os.fsencode(path), capi.ptr(sig_arr), len(sig_arr), int(multiple),
                                                    block_size, filter, level, ctypes.byref(h)))
        self.handle = h
        self.path = path

    def close(self):
        if self.handle:
            capi.lib().pg_supertensor_writer_close(self.handle)
            self.handle = None

    def __del__(self):
        self.close()


class supertensor_writer_t:
    """Writer of one section (supertensor.h:176-215).  A file left without
    finalize() is removed when its writers are closed or collected."""

    def __init__(self, path, section, block_size=8, filter=1, level=6, _writer=None, _section=0):
        sig = section if isinstance(section, (int, np.integer)) else section_sig(section)
        self._w = _writer if _writer is not None else _Writer(path, [sig], False, block_size, filter, level)
        self._section = _section
        self.level = level
        shape = section_shape(int(sig))
        self.header = supertensor_header_t(_plain_header(int(sig), shape, block_size, filter))

    def write_block(self, block, data, turn=RAW, threads=0, stream=None):
        """Write one block from a device node tensor (shape block_shape + (8,))."""
        self.write_blocks([block], data, [0], turn, threads, stream)

    def write_blocks(self, blocks, nodes, node_offsets, turn=RAW, threads=0, stream=None):
        secs, b = _block_list([(self._section, blk) for blk in blocks])
        off = np.ascontiguousarray(node_offsets, dtype=np.int64)
        capi.check(capi.lib().pg_supertensor_write_blocks(self._w.handle, len(blocks), capi.ptr(secs), capi.ptr(b),
                                                          nodes.data_ptr(), capi.ptr(off), turn, threads,
                                                          capi.stream_handle(stream)))

    def write_block_filtered(self, block, data, threads=0):
        """Write one block from its on-disk (already filtered) bytes in host memory."""
        data = np.ascontiguousarray(np.frombuffer(bytes(data), np.uint8))
        secs, b = _block_list([(self._section, block)])
        off = np.zeros(1, np.int64)
        capi.check(capi.lib().pg_supertensor_write_blocks_host(self._w.handle, 1, capi.ptr(secs), capi.ptr(b),
                                                               capi.ptr(data), capi.ptr(off), threads))

    def finalize(self):
        capi.check(capi.lib().pg_supertensor_finalize(self._w.handle, self._section))

    def close(self):
        self._w.close()


def _plain_header(sig, shape, block_size, filter):
    h = capi.pg_supertensor_header_t()
    h.version = 3
    h.section = sig
    h.stones = sum(sum(c) for c in _counts(sig))
    h.block_size = block_size
    for i in range(4):
        h.shape[i] = shape[i]
        h.blocks[i] = (shape[i] + block_size - 1) // block_size
    h.filter = filter
    return h


def supertensor_writers(path, sections, block_size=8, filter=1, level=6):
    """One writer per section of a multiple-section file (supertensor.cc:437-464)."""
    sigs = [s if isinstance(s, (int, np.integer)) else section_sig(s) for s in sections]
    w = _Writer(path, sigs, True, block_size, filter, level)
    return [supertensor_writer_t(path, int(sig), block_size, filter, level, _writer=w, _section=i)
            for i, sig in enumerate(sigs)]


# ---------------------------------------------------------------------------
# Whole slices.  A slice tensor holds its sections (sorted by sig) back to
# back, each as 8^4 blocks in block-major order (pg_slice_layout); these map
# one to one onto the blocks of a supertensor file with block_size 8.

def section_block_offsets(shape):
    """Blocks of a section (row-major) and the node offset of each in the
    section's block-major layout."""
    shape = np.asarray(shape, np.int64)
    B = (shape + 7) // 8
    idx = np.stack(np.meshgrid(*[np.arange(b) for b in B], indexing="ij"), -1).reshape(-1, 4)
    bs = np.minimum(8, shape[None, :] - 8 * idx)
    off = np.zeros(len(idx), np.int64)
    before = np.ones(len(idx), np.int64)
    for i in range(4):
        after = int(np.prod(shape[i + 1:]))
        off += before * 8 * idx[:, i] * after
        before *= bs[:, i]
    return idx.astype(np.uint8), off


def _slice_blocks(sigs):
    from .sweep import slice_layout
    base = slice_layout(sigs)
    secs, blocks, offs = [], [], []
    for i, sig in enumerate(sigs):
        idx, off = section_block_offsets(section_shape(int(sig)))
        secs.append(np.full(len(idx), i, np.int32))
        blocks.append(idx)
        offs.append(off + base[i])
    return np.concatenate(secs), np.ascontiguousarray(np.concatenate(blocks)), np.concatenate(offs), int(base[-1])


def write_slice(path, slice_, sigs, nodes, level=6, threads=0, stream=None):
    """Write a slice tensor (end-engine node form, sections `sigs` sorted) as a
    multiple-section file: block size 8, interleave filter, on-disk pairs."""
    sigs = np.ascontiguousarray(sigs, dtype=np.uint64)
    secs, blocks, offs, total = _slice_blocks(sigs)
    if nodes.shape[0] != total:
        raise ValueError(f"slice tensor has {nodes.shape[0]} nodes, the sections {total}")
    w = _Writer(path, sigs, True, 8, 1, level)
    capi.check(capi.lib().pg_supertensor_write_blocks(w.handle, len(secs), capi.ptr(secs), capi.ptr(blocks),
                                                      nodes.data_ptr(), capi.ptr(offs), slice_ & 1, threads,
                                                      capi.stream_handle(stream)))
    capi.check(capi.lib().pg_supertensor_finalize(w.handle, -1))
    w.close()


class slice_writer:
    """A slice file written one section at a time (the same file write_slice
    makes): write_section(i, nodes of section i alone), then finalize()."""

    def __init__(self, path, slice_, sigs, level=6, threads=0):
        self.sigs = np.ascontiguousarray(sigs, dtype=np.uint64)
        self.turn = slice_ & 1
        self.threads = threads
        self._w = _Writer(path, self.sigs, True, 8, 1, level)

    def write_section(self, i, nodes, stream=None):
        idx, off = section_block_offsets(section_shape(int(self.sigs[i])))
        secs = np.full(len(idx), i, np.int32)
        blocks = np.ascontiguousarray(idx, dtype=np.uint8)
        offs = np.ascontiguousarray(off, dtype=np.int64)
        capi.check(capi.lib().pg_supertensor_write_blocks(self._w.handle, len(secs), capi.ptr(secs), capi.ptr(blocks),
                                                          nodes.data_ptr(), capi.ptr(offs), self.turn, self.threads,
                                                          capi.stream_handle(stream)))

    def finalize(self):
        capi.check(capi.lib().pg_supertensor_finalize(self._w.handle, -1))
        self._w.close()


def read_slice(path, sigs=None, threads=0, stream=None, out=None):
    """Read sections of a slice file into a slice tensor (end-engine node
    form).  sigs: the sections wanted (default: all in the file), sorted.
    out: a contiguous (nodes, 8) int64 device tensor to read into (default:
    a new one).  Returns (slice, sigs, tensor)."""
    import torch
    f = _File(path)
    headers = [supertensor_header_t(f.header(s)) for s in range(f.sections)]
    where = {h.section: i for i, h in enumerate(headers)}
    if sigs is None:
        sigs = np.array(sorted(where), np.uint64)
    sigs = np.ascontiguousarray(sigs, dtype=np.uint64)
    missing = [int(s) for s in sigs if int(s) not in where]
    if missing:
        raise KeyError(f"sections {missing} are not in {path}")
    stones = {headers[where[int(s)]].stones for s in sigs}
    if len(stones) != 1 or any(headers[where[int(s)]].block_size != 8 for s in sigs):
        raise ValueError("a slice file holds sections of one slice with block size 8")
    slice_ = stones.pop()
    secs, blocks, offs, total = _slice_blocks(sigs)
    file_secs = np.array([where[int(sigs[i])] for i in secs], np.int32)
    if out is None:
        out = torch.empty((total, 8), dtype=torch.int64, device="cuda")
    elif (tuple(out.shape) != (total, 8) or out.dtype != torch.int64 or not out.is_cuda
          or not out.is_contiguous()):
        raise ValueError(f"out must be a contiguous ({total}, 8) int64 device tensor")
    capi.check(capi.lib().pg_supertensor_read_blocks(f.handle, len(file_secs), capi.ptr(file_secs),
                                                     capi.ptr(blocks), out.data_ptr(), capi.ptr(offs), slice_ & 1,
                                                     threads, capi.stream_handle(stream)))
    f.close()
    return slice_, sigs, out


# ---------------------------------------------------------------------------
# Slice index files (.pentago.index, pentago/high/index.h, index.cc)
#
# A 20-byte magic, the slice (u32), then for every section of the slice in
# descendent_sections(empty board, slice) order and every block of it in
# row-major order a 12-byte blob: the block's file offset (u64, as two u32
# words, low first) and compressed size (u32), all little endian.  A reader
# with random access to the .pentago file fetches a block's blob at a
# computable offset, then the block's bytes.

INDEX_MAGIC = b"pentago index      \n"
INDEX_HEAD = 24
INDEX_BLOB = 12


def index_sections(slice_):
    """Every section of a slice in the index order (all sections reachable
    from the empty board, sorted as descendent_sections sorts them)."""
    from .sweep import descendent_sections
    return descendent_sections(0, slice_)


def _section_block_counts(sigs):
    return [int(np.prod((np.asarray(section_shape(int(s)), np.int64) + 7) // 8)) for s in sigs]


def write_index(path, slice_paths):
    """Write the .pentago.index of a complete slice held in the given slice
    files (write_supertensor_index, pentago/high/index.cc:82-118): every
    section of the slice must be in some file, with block size 8 and the
    interleave filter.  Returns the index bytes."""
    if isinstance(slice_paths, (str, bytes, os.PathLike)):
        slice_paths = [slice_paths]
    readers = {}
    slice_ = None
    for p in slice_paths:
        for r in open_supertensors(p):
            if r.header.filter != 1 or r.header.block_size != 8:
                raise ValueError("an index covers interleave-filtered files of block size 8")
            if slice_ is None:
                slice_ = r.header.stones
            elif r.header.stones != slice_:
                raise ValueError("the files hold more than one slice")
            readers[int(r.header.section)] = r
    if slice_ is None:
        raise ValueError("no sections")
    sigs = index_sections(slice_)
    missing = [int(s) for s in sigs if int(s) not in readers]
    if missing:
        raise KeyError(f"the slice's sections {missing} are in none of the files")
    parts = [INDEX_MAGIC, struct.pack("<I", slice_)]
    for sig in sigs:
        r = readers[int(sig)]
        for b in r.header.all_blocks():
            _, size, offset = r.blob(b)
            parts.append(struct.pack("<III", offset & 0xffffffff, offset >> 32, size))
    data = b"".join(parts)
    assert len(data) == INDEX_HEAD + INDEX_BLOB * sum(_section_block_counts(sigs))
    with open(path, "wb") as f:
        f.write(data)
    return data


@functools.lru_cache(maxsize=64)
def _index_layout(slice_):
    """Per section of a slice (in index order): its position and the number
    of blocks before it (the reference's section_offset, index.cc:22-33)."""
    sigs = index_sections(slice_)
    before = np.zeros(len(sigs) + 1, np.int64)
    before[1:] = np.cumsum(_section_block_counts(sigs))
    return {int(s): i for i, s in enumerate(sigs)}, before


def index_blob_location(slice_, section, block):
    """(offset, size) of a block's blob in the slice's index file
    (supertensor_index_t::blob_location, index.cc:48-59)."""
    where, before = _index_layout(int(slice_))
    if int(section) not in where:
        raise KeyError(f"section {section:#x} is not in slice {slice_}")
    i = where[int(section)]
    B = (np.asarray(section_shape(int(section)), np.int64) + 7) // 8
    if any(not 0 <= int(block[k]) < int(B[k]) for k in range(4)):
        raise IndexError(f"block {tuple(block)} outside {tuple(B)}")
    flat = int(np.ravel_multi_index(tuple(int(x) for x in block), tuple(int(x) for x in B)))
    return INDEX_HEAD + INDEX_BLOB * (int(before[i]) + flat), INDEX_BLOB


def index_block_location(blob):
    """(offset, compressed size) of a block in the .pentago file from its
    12-byte blob (supertensor_index_t::block_location, index.cc:61-67)."""
    blob = bytes(blob)
    if len(blob) != INDEX_BLOB:
        raise ValueError(f"expected {INDEX_BLOB} bytes, got {len(blob)}")
    lo, hi, size = struct.unpack("<III", blob)
    return lo | hi << 32, size


def index_read_block_filtered(pentago_path, index_data, slice_, section, block, expected_size=None):
    """A block's decompressed on-disk bytes (filtered as stored), fetched the
    way a byte-range reader does: its blob from the index, then its bytes
    from the .pentago file (supertensor_index_t::unpack_block's decompress,
    index.cc:69-74; xz streams are told from zlib ones by the xz magic, as
    pentago/data/compress.cc:37-40 does).  The GPU unfilter
    (pg_supertensor_unfilter) turns them into nodes."""
    import lzma
    import zlib
    off, size = index_blob_location(slice_, section, block)
    offset, csize = index_block_location(bytes(index_data[off:off + size]))
    with open(pentago_path, "rb") as f:
        f.seek(offset)
        raw = f.read(csize)
    if len(raw) != csize:
        raise IOError(f"{pentago_path}: block {tuple(block)} of section {section:#x} is truncated")
    data = lzma.decompress(raw) if raw[:6] == b"\xfd7zXZ\x00" else zlib.decompress(raw)
    if expected_size is not None and len(data) != expected_size:
        raise ValueError(f"block {tuple(block)}: {len(data)} bytes, expected {expected_size}")
    return np.frombuffer(data, np.uint8)


# ---------------------------------------------------------------------------
# Measurement

IO_ROOT = [[4, 4], [5, 4], [4, 5], [4, 3]]   # a 33-stone root: its slice 34 is 2.7 GB of solved nodes


def bench_filter(nodes=1 << 24, reps=5):
    """Filter and unfilter kernels alone: 64 B read + 64 B written per node,
    inputs and outputs (1 GiB each at the default size) far beyond L2."""
    import torch
    L = capi.lib()
    a = torch.randint(-2**62, 2**62, (nodes, 8), dtype=torch.int64, device="cuda")
    b = torch.empty_like(a)
    s = capi.stream_handle()
    out = {}
    for name, f, src, dst in (("filter", L.pg_supertensor_filter, a, b), ("unfilter", L.pg_supertensor_unfilter, b, a)):
        for _ in range(2):
            capi.check(f(src.data_ptr(), nodes, 0, 1, dst.data_ptr(), s))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            capi.check(f(src.data_ptr(), nodes, 0, 1, dst.data_ptr(), s))
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        out[name] = {"ms": ms, "GBps": 128 * nodes / (ms / 1e3) / 1e9}
    out["nodes"] = nodes
    out["bytes_per_node"] = 128
    return out


def bench_slice_io(levels=(1, 6), threads=0, directory=None):
    """Write and read back a real solved slice (slice 34 below IO_ROOT) with
    the GPU filter and host-thread compression; wall-clock GB/s of node data."""
    import shutil
    import tempfile
    import time
    import torch
    from . import sweep as sweep_mod
    root = section_sig(IO_ROOT)
    _, nodes, sigs = sweep_mod.sweep(root, min_slice=34, keep_last=True)
    torch.cuda.synchronize()
    nbytes = nodes.shape[0] * 64
    d = tempfile.mkdtemp(dir=directory)
    res = {"workload": f"slice 34 below the root {IO_ROOT}: {len(sigs)} sections, {nodes.shape[0]} nodes "
                       f"({nbytes / 1e9:.2f} GB), block size 8, interleave filter",
           "threads": threads or os.cpu_count(), "levels": {}}
    try:
        for level in levels:
            path = os.path.join(d, f"slice-34-{level}.pentago")
            t = time.perf_counter()
            write_slice(path, 34, sigs, nodes, level=level, threads=threads)
            tw = time.perf_counter() - t
            size = os.path.getsize(path)
            t = time.perf_counter()
            _, _, back = read_slice(path, threads=threads)
            torch.cuda.synchronize()
            tr = time.perf_counter() - t
            ok = bool(torch.equal(back, nodes))
            del back
            res["levels"][str(level)] = {"write_s": tw, "read_s": tr, "write_GBps": nbytes / tw / 1e9,
                                         "read_GBps": nbytes / tr / 1e9, "file_bytes": size,
                                         "bits_per_position": 8 * size / (nodes.shape[0] * 256), "roundtrip_ok": ok}
            os.remove(path)
    finally:
        shutil.rmtree(d, ignore_errors=True)
    return res


def main():
    import argparse
    import json
    ap = argparse.ArgumentParser(description="slice-file filter and I/O throughput")
    ap.add_argument("--threads", type=int, default=0)
    ap.add_argument("--levels", default="1,6")
    args = ap.parse_args()
    import torch
    capi.check(capi.lib().pg_init())
    torch.zeros(1, device="cuda")
    print(json.dumps({"filter_kernels": bench_filter(),
                      "slice_io": bench_slice_io(tuple(int(x) for x in args.levels.split(",")), args.threads)}))


if __name__ == "__main__":
    main()
