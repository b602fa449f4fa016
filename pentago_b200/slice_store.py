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
