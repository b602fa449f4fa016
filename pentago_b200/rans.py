"""rANS coding of solved blocks: the GPU static coder (format version 2 of
pentago/shard/arithmetic.cc, byte-identical) and the learned coder built on it.

``encode(streams)`` / ``decode(blobs)`` take and return lists of host arrays;
``encode_device`` / ``decode_device`` keep everything on the GPU.
"""
import numpy as np

from . import capi


def bound(n):
    return int(capi.lib().pg_rans_bound(int(n)))


def _align(x, a=256):
    return (x + a - 1) // a * a


def encode_device(symbols, offsets, stream=None):
    """symbols: device uint8 tensor; offsets: host int64 array of stream bounds.
    Returns (device output bytes, host out_offsets, host sizes)."""
    import torch
    offsets = np.ascontiguousarray(offsets, dtype=np.int64)
    ns = len(offsets) - 1
    caps = [_align(bound(offsets[i + 1] - offsets[i])) for i in range(ns)]
    out_off = np.zeros(ns + 1, np.int64)
    out_off[1:] = np.cumsum(caps)
    dev = symbols.device
    out = torch.empty(int(out_off[-1]) or 1, dtype=torch.uint8, device=dev)
    d_off = torch.from_numpy(offsets).to(dev)
    d_oo = torch.from_numpy(out_off[:-1].copy()).to(dev)
    sizes = torch.zeros(max(ns, 1), dtype=torch.int64, device=dev)
    capi.check(capi.lib().pg_rans_encode_batch(symbols.data_ptr(), d_off.data_ptr(), ns, out.data_ptr(),
                                               d_oo.data_ptr(), sizes.data_ptr(), capi.stream_handle(stream)))
    sz = sizes.cpu().numpy()[:ns]
    if (sz < 0).any():
        raise capi.PentagoError(int(sz.min()), "invalid symbols (values must be 0, 1 or 2)")
    return out, out_off, sz


def decode_device(data, in_offsets, in_sizes, sym_offsets, stream=None):
    """data: device uint8 tensor of streams.  Returns (device symbols, host status)."""
    import torch
    ns = len(in_sizes)
    dev = data.device
    sym_offsets = np.ascontiguousarray(sym_offsets, dtype=np.int64)
    caps = np.diff(sym_offsets).astype(np.int64)
    symbols = torch.empty(int(sym_offsets[-1]) or 1, dtype=torch.uint8, device=dev)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.int64)).to(dev)
    d_in, d_sz, d_so, d_cap = t(in_offsets[:ns]), t(in_sizes), t(sym_offsets[:ns]), t(caps)
    status = torch.zeros(max(ns, 1), dtype=torch.int64, device=dev)
    capi.check(capi.lib().pg_rans_decode_batch(data.data_ptr(), d_in.data_ptr(), d_sz.data_ptr(), ns,
                                               symbols.data_ptr(), d_so.data_ptr(), d_cap.data_ptr(),
                                               status.data_ptr(), capi.stream_handle(stream)))
    return symbols, status.cpu().numpy()[:ns]


def encode(streams):
    """List of host uint8 symbol arrays -> list of serialized v2 streams (bytes)."""
    import torch
    lens = [len(s) for s in streams]
    offsets = np.zeros(len(streams) + 1, np.int64)
    offsets[1:] = np.cumsum(lens)
    flat = np.concatenate([np.asarray(s, np.uint8) for s in streams]) if streams else np.zeros(0, np.uint8)
    sym = torch.from_numpy(flat if len(flat) else np.zeros(1, np.uint8)).cuda()
    out, out_off, sizes = encode_device(sym, offsets)
    host = out.cpu().numpy()
    return [host[out_off[i]:out_off[i] + sizes[i]].tobytes() for i in range(len(streams))]


def decode(blobs, counts=None):
    """List of serialized streams -> list of host uint8 symbol arrays.  Raises
    on malformed streams (PG_ERR_FORMAT)."""
    import torch
    sizes = np.array([len(b) for b in blobs], np.int64)
    in_off = np.zeros(len(blobs) + 1, np.int64)
    in_off[1:] = np.cumsum([_align(len(b), 16) for b in blobs])
    buf = np.zeros(int(in_off[-1]) or 1, np.uint8)
    for i, b in enumerate(blobs):
        buf[in_off[i]:in_off[i] + len(b)] = np.frombuffer(b, np.uint8)
    if counts is None:
        counts = [int(np.frombuffer(b[4:28], "<u8").sum()) if len(b) >= 28 else 0 for b in blobs]
    so = np.zeros(len(blobs) + 1, np.int64)
    so[1:] = np.cumsum(counts)
    syms, status = decode_device(torch.from_numpy(buf).cuda(), in_off, sizes, so)
    if (status < 0).any():
        raise capi.PentagoError(int(status.min()), "malformed rANS stream")
    host = syms.cpu().numpy()
    return [host[so[i]:so[i] + status[i]] for i in range(len(blobs))]


def node_symbols(nodes, turn, stream=None):
    """Device (n, 8) int64 nodes -> device uint8 symbols (256 per node)."""
    import torch
    n = nodes.shape[0]
    out = torch.empty(max(256 * n, 1), dtype=torch.uint8, device=nodes.device)
    capi.check(capi.lib().pg_node_symbols(nodes.data_ptr(), n, turn, out.data_ptr(), capi.stream_handle(stream)))
    return out[:256 * n]
