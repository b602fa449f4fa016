"""A solved slice kept compressed in HBM, so that a sweep can go deeper.

The role of the reference's in-memory block compression
(pentago/end/fast_compress.cc, compacting_store.cc) for the GPU sweep: every
8^4 block of a slice is coded by the library's store coder (pg_store_*: rANS
with a 1024-context model of each rotation's neighbours, one frequency table
per chunk of blocks, coded from and decoded to nodes on the GPU), and a child
section is decompressed into a staging buffer only while the lines that read
it run (pg_end_sweep_slice_child).  A slice then costs its coded size while
the slice below it is built.
"""
import numpy as np

from . import capi
from .end import section_shape


def slice_blocks(sigs):
    """Every block of a slice in memory order: (section index, first node,
    node count) arrays, each section's first block, and the section bases."""
    from .sweep import slice_layout
    from .supertensor import section_block_offsets
    base = slice_layout(sigs)
    sec, first, count, sec_first = [], [], [], [0]
    for i, sig in enumerate(sigs):
        shape = np.array(section_shape(int(sig)), np.int64)
        idx, off = section_block_offsets(shape)
        sec.append(np.full(len(idx), i, np.int32))
        first.append(off + base[i])
        count.append(np.minimum(8, shape[None, :] - 8 * idx.astype(np.int64)).prod(1))
        sec_first.append(sec_first[-1] + len(idx))
    return np.concatenate(sec), np.concatenate(first), np.concatenate(count), np.array(sec_first), base


# The store coder's streams: LANES lanes per block, a header of their lengths.
LANES = 32
HEAD = 4 * LANES


def store_bound(count):
    """pg_store_bound for an array of block node counts: the header and LANES
    lanes of the raw size of ceil(count / LANES) nodes plus 64 bytes each."""
    count = np.asarray(count, np.int64)
    return HEAD + LANES * ((count + LANES - 1) // LANES * 64 + 64)


class compressed_slice:
    """A slice tensor (end-engine nodes, sections `sigs` in slice layout) as
    one store-coder stream per block, in chunks of at most chunk_nodes nodes
    (one frequency table and one packed byte buffer per chunk)."""

    def __init__(self, nodes, sigs, turn, chunk_nodes=1 << 26, stream=None):
        """Code a whole slice tensor (nodes None: start empty and add sections)."""
        self.sigs = np.ascontiguousarray(sigs, dtype=np.uint64)
        self.turn = turn
        self.chunk_nodes = chunk_nodes
        self.sec, self.first, self.count, self.sec_first, self.base = slice_blocks(self.sigs)
        self.raw_bytes = 64 * int(self.base[-1])
        self.chunks = []   # (first block, last block + 1, table, device bytes, packed offsets, sizes)
        self.bytes = 0
        if nodes is not None:
            for i in range(len(self.sigs)):
                self.add_section(i, nodes[int(self.base[i]):int(self.base[i + 1])], stream)

    def add_section(self, i, nodes, stream=None):
        """Code section i from its nodes (block-major, the section alone)."""
        import torch
        L = capi.lib()
        sh = capi.stream_handle(stream)
        dev = nodes.device
        t64 = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.int64)).to(dev)
        lo, hi = int(self.sec_first[i]), int(self.sec_first[i + 1])
        n_base = int(self.base[i])
        b0 = lo
        while b0 < hi:
            b1, used = b0, 0
            while b1 < hi and (b1 == b0 or used + self.count[b1] <= self.chunk_nodes):
                used += int(self.count[b1])
                b1 += 1
            k = b1 - b0
            first = t64(self.first[b0:b1] - n_base)
            count = torch.from_numpy(self.count[b0:b1].astype(np.int32)).to(dev)
            table = torch.empty(1024 * 3, dtype=torch.int16, device=dev)
            capi.check(L.pg_store_table(nodes.data_ptr(), first.data_ptr(), count.data_ptr(), k, self.turn,
                                        table.data_ptr(), sh))
            caps = (store_bound(self.count[b0:b1]) + 15) // 16 * 16
            out_off = np.zeros(k + 1, np.int64)
            out_off[1:] = np.cumsum(caps)
            out = torch.empty(int(out_off[-1]), dtype=torch.uint8, device=dev)
            d_off = t64(out_off[:-1])
            sizes = torch.zeros(k, dtype=torch.int64, device=dev)
            capi.check(L.pg_store_encode(nodes.data_ptr(), first.data_ptr(), count.data_ptr(), k, self.turn,
                                         table.data_ptr(), out.data_ptr(), d_off.data_ptr(), sizes.data_ptr(), sh))
            sz = sizes.cpu().numpy()
            # the coder leaves room for its worst case after every stream: pack
            # them, each starting on a 16-byte boundary
            packed = np.zeros(k + 1, np.int64)
            packed[1:] = np.cumsum((sz + 15) // 16 * 16)
            data = torch.empty(max(int(packed[-1]), 1), dtype=torch.uint8, device=dev)
            d_packed = t64(packed[:-1])
            capi.check(L.pg_pack_streams(out.data_ptr(), d_off.data_ptr(), sizes.data_ptr(), k, data.data_ptr(),
                                         d_packed.data_ptr(), sh))
            del out
            self.chunks.append((b0, b1, table, data, packed, sz.astype(np.int64)))
            self.bytes += int(data.numel()) + 2 * 1024 * 3
            b0 = b1

    def section_nodes(self, i, stream=None):
        """Section i's nodes (block-major), decompressed on the GPU."""
        import torch
        L = capi.lib()
        lo, hi = int(self.sec_first[i]), int(self.sec_first[i + 1])
        n_base = int(self.base[i])
        out = torch.empty((int(self.base[i + 1]) - n_base, 8), dtype=torch.int64, device="cuda")
        t64 = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.int64)).to(out.device)
        for b0, b1, table, data, packed, sz in self.chunks:
            a, b = max(lo, b0), min(hi, b1)
            if a >= b:
                continue
            k0, k1 = a - b0, b - b0
            count = torch.from_numpy(self.count[a:b].astype(np.int32)).to(out.device)
            status = torch.zeros(k1 - k0, dtype=torch.int64, device=out.device)
            d_in, d_sz, d_dst = t64(packed[k0:k1]), t64(sz[k0:k1]), t64(self.first[a:b] - n_base)
            capi.check(L.pg_store_decode(data.data_ptr(), d_in.data_ptr(), d_sz.data_ptr(), count.data_ptr(),
                                         d_dst.data_ptr(), k1 - k0, self.turn, table.data_ptr(), out.data_ptr(),
                                         status.data_ptr(), capi.stream_handle(stream)))
            if (status.cpu().numpy() != self.count[a:b]).any():
                raise capi.PentagoError(capi.PG_ERR_FORMAT, "a compressed block did not decode")
        return out


# ---------------------------------------------------------------------------
# Measurement

TIMING_ROOT = [[4, 4], [4, 5], [4, 3], [3, 3]]   # its slice 33: 35.4 GB in 10 sections
SMALL_ROOT = [[4, 4], [5, 4], [4, 5], [4, 3]]    # its slice 34: 2.7 GB in 2 sections


def _coder_case(root, slice_, max_nodes, largest_section, reps):
    """Solve root's slices down to slice_, take a batch of at most max_nodes
    nodes of consecutive blocks (from the largest section, or from the slice's
    start), and time the table, encode and decode kernels on it with CUDA
    events (each run once untimed, then reps times); check the round trip."""
    import torch
    from . import sweep
    from .end import section_sig
    L = capi.lib()
    capi.check(L.pg_init())
    _, nodes, sigs = sweep.sweep(section_sig(root), min_slice=slice_, keep_last=True)
    _, first, count, sec_first, base = slice_blocks(sigs)
    dev = nodes.device
    i = int(np.argmax(np.diff(base))) if largest_section else 0
    lo, hi = (int(sec_first[i]), int(sec_first[i + 1])) if largest_section else (0, len(count))
    b1, used = lo, 0
    while b1 < hi and used + count[b1] <= max_nodes:
        used += int(count[b1])
        b1 += 1
    k = b1 - lo
    turn = slice_ & 1
    t64 = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.int64)).to(dev)
    d_first, d_count = t64(first[lo:b1]), torch.from_numpy(count[lo:b1].astype(np.int32)).to(dev)
    table = torch.empty(3 * 1024, dtype=torch.int16, device=dev)
    caps = (store_bound(count[lo:b1]) + 15) // 16 * 16
    off = np.zeros(k + 1, np.int64)
    off[1:] = np.cumsum(caps)
    out = torch.empty(int(off[-1]), dtype=torch.uint8, device=dev)
    d_off = t64(off[:-1])
    sizes = torch.zeros(k, dtype=torch.int64, device=dev)

    def timed(fn):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        fn()
        torch.cuda.synchronize()
        if not reps:
            return None
        a.record()
        for _ in range(reps):
            fn()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / reps

    ms_table = timed(lambda: capi.check(L.pg_store_table(nodes.data_ptr(), d_first.data_ptr(), d_count.data_ptr(),
                                                         k, turn, table.data_ptr(), None)))
    ms_encode = timed(lambda: capi.check(L.pg_store_encode(nodes.data_ptr(), d_first.data_ptr(), d_count.data_ptr(),
                                                           k, turn, table.data_ptr(), out.data_ptr(), d_off.data_ptr(),
                                                           sizes.data_ptr(), None)))
    sz = sizes.cpu().numpy()
    dst = torch.empty((used, 8), dtype=torch.int64, device=dev)
    status = torch.zeros(k, dtype=torch.int64, device=dev)
    d_sz, d_dst = t64(sz), t64(first[lo:b1] - first[lo])
    ms_decode = timed(lambda: capi.check(L.pg_store_decode(out.data_ptr(), d_off.data_ptr(), d_sz.data_ptr(),
                                                           d_count.data_ptr(), d_dst.data_ptr(), k, turn,
                                                           table.data_ptr(), dst.data_ptr(), status.data_ptr(), None)))
    ok = bool(torch.equal(dst, nodes[int(first[lo]):int(first[lo]) + used]))
    symbols = used * 256
    rate = lambda ms: symbols / (ms / 1e3) / 1e9 if ms else None
    return {"root": root, "slice": slice_, "blocks": k, "nodes": used, "symbols": symbols,
            "ratio": 64 * used / float(sz.sum()), "ms": {"table": ms_table, "encode": ms_encode, "decode": ms_decode},
            "G_symbols_per_s": {"table": rate(ms_table), "encode": rate(ms_encode), "decode": rate(ms_decode)},
            "roundtrip": ok}


def main():
    """Store-coder kernels on one batch of a solved slice.

        python -m pentago_b200.slice_store           # 2^26 nodes of the largest
                                                     # section of slice 33 of
                                                     # [[4,4],[4,5],[4,3],[3,3]]
        python -m pentago_b200.slice_store --small   # 2^24 nodes of slice 34 of
                                                     # [[4,4],[5,4],[4,5],[4,3]],
                                                     # each kernel once (profiling)
    """
    import argparse
    import json
    ap = argparse.ArgumentParser(description="store-coder kernels on one batch of a solved slice")
    ap.add_argument("--small", action="store_true", help="the small case: few GB on the device, one run per kernel")
    args = ap.parse_args()
    if args.small:
        res = _coder_case(SMALL_ROOT, 34, 1 << 24, largest_section=False, reps=0)
    else:
        res = _coder_case(TIMING_ROOT, 33, 1 << 26, largest_section=True, reps=3)
    print(json.dumps(res))
    if not res["roundtrip"]:
        raise SystemExit("store coder round trip failed")


if __name__ == "__main__":
    main()
