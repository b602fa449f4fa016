"""A solved slice kept compressed in HBM, so that a sweep can go deeper.

The role of the reference's in-memory block compression
(pentago/end/fast_compress.cc, compacting_store.cc) for the GPU sweep: every
8^4 block of a slice becomes one format-2 rANS stream (the reference's own
coder, byte-identical, on the GPU) of its 256 symbols per node, and a child
section is decompressed into a staging buffer only while the lines that read
it run (pg_end_sweep_slice_child).  A slice then costs its coded size while
the slice below it is built.
"""
import numpy as np

from . import capi, rans
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


class compressed_slice:
    """A slice tensor (end-engine nodes, sections `sigs` in slice layout) as
    one format-2 stream per block, coded in chunks of at most chunk_nodes
    nodes and packed back to back per chunk."""

    def __init__(self, nodes, sigs, turn, chunk_nodes=1 << 24, stream=None):
        import torch
        self.sigs = np.ascontiguousarray(sigs, dtype=np.uint64)
        self.turn = turn
        self.sec, self.first, self.count, self.sec_first, self.base = slice_blocks(self.sigs)
        self.raw_bytes = 64 * int(self.base[-1])
        self.chunks = []   # (first block, last block + 1, device bytes, packed stream offsets, sizes)
        nb = len(self.first)
        b0 = 0
        while b0 < nb:
            b1, used = b0, 0
            while b1 < nb and (b1 == b0 or used + self.count[b1] <= chunk_nodes):
                used += int(self.count[b1])
                b1 += 1
            n0 = int(self.first[b0])
            sym = rans.node_symbols(nodes[n0:n0 + used], turn, stream)
            sym_off = np.zeros(b1 - b0 + 1, np.int64)
            sym_off[1:] = 256 * np.cumsum(self.count[b0:b1])
            out, out_off, sz = rans.encode_device(sym, sym_off, stream)
            del sym
            # the coder leaves room for its worst case after every stream: pack them
            dev = out.device
            packed = np.zeros(len(sz) + 1, np.int64)
            packed[1:] = np.cumsum(sz)
            data = torch.empty(max(int(packed[-1]), 1), dtype=torch.uint8, device=dev)
            t = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.int64)).to(dev)
            d_in, d_sz, d_out = t(out_off[:-1]), t(sz), t(packed[:-1])
            capi.check(capi.lib().pg_pack_streams(out.data_ptr(), d_in.data_ptr(), d_sz.data_ptr(), len(sz),
                                                  data.data_ptr(), d_out.data_ptr(), capi.stream_handle(stream)))
            del out
            self.chunks.append((b0, b1, data, packed, sz.astype(np.int64)))
            b0 = b1
        self.bytes = sum(int(c[2].numel()) for c in self.chunks)

    def section_nodes(self, i, stream=None):
        """Section i's nodes (block-major), decompressed on the GPU."""
        import torch
        lo, hi = int(self.sec_first[i]), int(self.sec_first[i + 1])
        n_base = int(self.base[i])
        out = torch.empty((int(self.base[i + 1]) - n_base, 8), dtype=torch.int64, device="cuda")
        for b0, b1, data, packed, sz in self.chunks:
            a, b = max(lo, b0), min(hi, b1)
            if a >= b:
                continue
            k0, k1 = a - b0, b - b0
            sym_off = np.zeros(k1 - k0 + 1, np.int64)
            sym_off[1:] = 256 * np.cumsum(self.count[a:b])
            sym, status = rans.decode_device(data, packed[k0:k1 + 1], sz[k0:k1], sym_off, stream)
            if (status != 256 * self.count[a:b]).any():
                raise capi.PentagoError(capi.PG_ERR_FORMAT, "a compressed block did not decode")
            n0 = int(self.first[a]) - n_base
            n = int(self.count[a:b].sum())
            capi.check(capi.lib().pg_symbols_nodes(sym.data_ptr(), n, self.turn, out[n0:n0 + n].data_ptr(),
                                                   capi.stream_handle(stream)))
            del sym
        return out
