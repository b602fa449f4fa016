"""Learned-model rANS for solved blocks (stream format version 3).

A 3-layer MLP (hidden 64, bf16 weights, fp32 arithmetic) predicts each
ternary symbol of a block (pg_node_symbols' convention, 256 rotations per
node) from the node's board, the rotation and the already coded neighbouring
rotations; the rANS coder codes with those probabilities.  The network is
trained on the GPU by the library's own kernels (pg_learned_grad /
pg_learned_adam) on a seeded subset of the blocks to be coded, serialized
with pg_learned_export, and the same bytes drive encoder and decoder.  The
encoder keeps the format-2 stream (the reference's coder,
pentago/shard/arithmetic.cc:366-495) for any block where it is smaller.

    python -m pentago_b200.learned --root 4,4,4,5,4,3,3,3

solves the root's sections down to its own slice, trains on 1% of the root
slice's blocks, codes every block of that slice both ways and prints one
JSON line (bits per position, GB/s, lossless check).
"""
import argparse
import ctypes
import json
import math
import time

import numpy as np

from . import capi

N_PARAMS = 12355  # W1 124x64, b1, W2 64x64, b2, W3 64x3, b3
P_W1, P_B1, P_W2, P_B2, P_W3, P_B3 = 0, 7936, 8000, 12096, 12160, 12352


def model_bytes():
    return int(capi.lib().pg_learned_model_bytes())


def _counts(sig):
    return [[(int(sig) >> (16 * q + 8 * k)) & 255 for k in range(2)] for q in range(4)]


def section_blocks(sig, shape):
    """Blocks of one section in slice order: (block coords (m, 4), node counts, node offsets)."""
    S = np.asarray(shape, np.int64)
    G = (S + 7) // 8
    b = np.stack(np.meshgrid(*[np.arange(g) for g in G], indexing="ij"), -1).reshape(-1, 4)
    bs = np.minimum(8, S[None, :] - 8 * b)
    off = np.zeros(len(b), np.int64)
    before = np.ones(len(b), np.int64)
    for i in range(4):
        after = int(np.prod(S[i + 1:]))
        off += before * 8 * b[:, i] * after
        before *= bs[:, i]
    return b, bs.prod(1), off


def slice_blocks(sigs, layout):
    """All blocks of a slice tensor: (pg_block_ref_t array, node offset of each block, nodes per block)."""
    from .end import section_shape
    refs, offs, counts = [], [], []
    for sig, base in zip(sigs, layout[:-1]):
        b, n, off = section_blocks(sig, section_shape(int(sig)))
        refs.append((int(sig), b))
        offs.append(int(base) + off)
        counts.append(n)
    total = sum(len(b) for _, b in refs)
    arr = (capi.pg_block_ref_t * total)()
    k = 0
    for sig, b in refs:
        for row in b:
            arr[k].section = sig
            for q in range(4):
                arr[k].block[q] = int(row[q])
            k += 1
    return arr, np.concatenate(offs), np.concatenate(counts)


def subset(refs, indices):
    out = (capi.pg_block_ref_t * len(indices))()
    for j, i in enumerate(indices):
        out[j] = refs[int(i)]
    return out


def block_symbols(slice_t, node_off, nodes, turn, stream=None):
    """Symbols of the given blocks of a slice tensor, concatenated: (device uint8, device offsets)."""
    import torch
    from . import rans
    idx = torch.cat([torch.arange(int(o), int(o) + int(n), device=slice_t.device) for o, n in zip(node_off, nodes)])
    sym = rans.node_symbols(slice_t[idx].contiguous(), turn, stream)
    offsets = torch.zeros(len(nodes) + 1, dtype=torch.int64)
    offsets[1:] = torch.from_numpy(np.cumsum(np.asarray(nodes, np.int64) * 256))
    return sym, offsets.to(slice_t.device)


def init_params(seed=0):
    """Initial fp32 parameters (device)."""
    import torch
    g = torch.Generator().manual_seed(seed)
    p = torch.zeros(N_PARAMS)
    p[P_W1:P_B1] = torch.randn(P_B1 - P_W1, generator=g) * 0.15
    p[P_W2:P_B2] = torch.randn(P_B2 - P_W2, generator=g) * math.sqrt(2 / 64)
    p[P_W3:P_B3] = torch.randn(P_B3 - P_W3, generator=g) * 0.1
    return p.cuda()


class Trainer:
    """Adam on the summed cross entropy of seeded sample batches, all on the GPU."""

    def __init__(self, refs, symbols, offsets, nodes, seed=0, params=None, stream=None):
        import torch
        self.refs, self.symbols, self.offsets = refs, symbols, offsets
        self.params = init_params(seed) if params is None else params.clone()
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.grad = torch.zeros_like(self.params)
        self.loss = torch.zeros(1, dtype=torch.float32, device="cuda")
        cand = [(s << 16) | np.arange(int(n), dtype=np.int64) for s, n in enumerate(nodes)]
        self.cand = torch.from_numpy(np.concatenate(cand)).cuda()
        self.seed = seed
        self.step = 0
        self.stream = capi.stream_handle(stream)
        self.samples = None

    def grad_of(self, samples):
        L = capi.lib()
        capi.check(L.pg_learned_grad(self.params.data_ptr(), self.refs, len(self.refs), self.symbols.data_ptr(),
                                     self.offsets.data_ptr(), samples.data_ptr(), samples.numel(),
                                     self.grad.data_ptr(), self.loss.data_ptr(), self.stream))
        return self.grad, self.loss

    def run(self, steps, batch=32768, lr=3e-3, lr_min=2e-4, log_every=0):
        import torch
        L = capi.lib()
        if self.samples is None or self.samples.numel() != batch:
            self.samples = torch.empty(batch, dtype=torch.int64, device="cuda")
        history = []
        for t in range(steps):
            self.step += 1
            capi.check(L.pg_learned_samples(self.cand.data_ptr(), self.cand.numel(), ctypes.c_uint64(self.seed),
                                            self.step, batch, self.samples.data_ptr(), self.stream))
            self.grad_of(self.samples)
            rate = lr_min + 0.5 * (lr - lr_min) * (1 + math.cos(math.pi * t / max(1, steps - 1)))
            capi.check(L.pg_learned_adam(self.params.data_ptr(), self.m.data_ptr(), self.v.data_ptr(),
                                         self.grad.data_ptr(), self.step, ctypes.c_float(rate),
                                         ctypes.c_float(1.0 / batch), self.stream))
            if log_every and (t % log_every == 0 or t == steps - 1):
                history.append((t, float(self.loss.item()) / batch))
        return history

    def model(self):
        return export(self.params)


def export(params):
    p = np.ascontiguousarray(params.detach().float().cpu().numpy())
    out = np.zeros(model_bytes(), np.uint8)
    capi.check(capi.lib().pg_learned_export(capi.ptr(p), capi.ptr(out)))
    return out.tobytes()


def _model_ptr(model):
    return ctypes.create_string_buffer(bytes(model), len(model))


def encode(model, refs, symbols, offsets, nodes, stream=None):
    """Code each block; returns (device stream bytes, device offsets, host sizes)."""
    import torch
    L = capi.lib()
    nodes = np.asarray(nodes, np.int64)
    caps = np.array([L.pg_rans_learned_bound(int(n)) for n in nodes], np.int64)
    out_off = np.zeros(len(nodes) + 1, np.int64)
    out_off[1:] = np.cumsum((caps + 15) // 16 * 16)
    out = torch.empty(int(out_off[-1]), dtype=torch.uint8, device="cuda")
    out_off_d = torch.from_numpy(out_off).cuda()
    sizes = torch.empty(len(nodes), dtype=torch.int64, device="cuda")
    m = _model_ptr(model)
    capi.check(L.pg_rans_learned_encode(m, refs, len(refs), symbols.data_ptr(), offsets.data_ptr(), out.data_ptr(),
                                        out_off_d.data_ptr(), sizes.data_ptr(), capi.stream_handle(stream)))
    return out, out_off_d, sizes


def decode(model, refs, data, in_offsets, in_sizes, nodes, stream=None):
    """Decode each block; returns (device symbols, device offsets, host status)."""
    import torch
    L = capi.lib()
    nodes = np.asarray(nodes, np.int64)
    sym_off = np.zeros(len(nodes) + 1, np.int64)
    sym_off[1:] = np.cumsum(nodes * 256)
    symbols = torch.empty(max(int(sym_off[-1]), 1), dtype=torch.uint8, device="cuda")
    caps = torch.from_numpy(nodes * 256).cuda()
    sym_off_d = torch.from_numpy(sym_off).cuda()
    status = torch.empty(len(nodes), dtype=torch.int64, device="cuda")
    m = _model_ptr(model)
    capi.check(L.pg_rans_learned_decode(m, refs, len(refs), data.data_ptr(), in_offsets.data_ptr(),
                                        in_sizes.data_ptr(), symbols.data_ptr(), sym_off_d.data_ptr(),
                                        caps.data_ptr(), status.data_ptr(), capi.stream_handle(stream)))
    return symbols[:int(sym_off[-1])], sym_off_d, status


def freqs(model, refs, symbols, offsets, samples, stream=None):
    import torch
    out = torch.empty((samples.numel(), 3), dtype=torch.int32, device="cuda")
    m = _model_ptr(model)
    capi.check(capi.lib().pg_learned_freqs(m, refs, len(refs), symbols.data_ptr(), offsets.data_ptr(),
                                           samples.data_ptr(), samples.numel(), out.data_ptr(),
                                           capi.stream_handle(stream)))
    return out


def static_roundtrip(symbols, offsets, stream=None):
    """Format-2 coding of the same symbol ranges on the GPU, timed both ways:
    (sizes, encode ms, decode ms, lossless)."""
    import torch
    L = capi.lib()
    off = offsets.cpu().numpy()
    n = len(off) - 1
    caps = np.array([L.pg_rans_bound(int(off[i + 1] - off[i])) for i in range(n)], np.int64)
    out_off = np.zeros(n + 1, np.int64)
    out_off[1:] = np.cumsum(caps)
    out = torch.empty(int(out_off[-1]), dtype=torch.uint8, device="cuda")
    out_off_d = torch.from_numpy(out_off).cuda()
    sizes = torch.empty(n, dtype=torch.int64, device="cuda")
    back = torch.empty_like(symbols)
    sym_caps = (offsets[1:] - offsets[:-1]).contiguous()
    status = torch.empty(n, dtype=torch.int64, device="cuda")
    h = capi.stream_handle(stream)
    e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    e0.record()
    capi.check(L.pg_rans_encode_batch(symbols.data_ptr(), offsets.data_ptr(), n, out.data_ptr(),
                                      out_off_d.data_ptr(), sizes.data_ptr(), h))
    e1.record()
    capi.check(L.pg_rans_decode_batch(out.data_ptr(), out_off_d.data_ptr(), sizes.data_ptr(), n, back.data_ptr(),
                                      offsets.data_ptr(), sym_caps.data_ptr(), status.data_ptr(), h))
    e2.record()
    torch.cuda.synchronize()
    ok = bool(torch.equal(back, symbols)) and bool(torch.equal(status, sym_caps))
    return sizes, e0.elapsed_time(e1), e1.elapsed_time(e2), ok


def static_sizes(symbols, offsets, stream=None):
    """Format-2 stream sizes of the same symbol ranges."""
    import torch
    L = capi.lib()
    off = offsets.cpu().numpy()
    n = len(off) - 1
    caps = np.array([L.pg_rans_bound(int(off[i + 1] - off[i])) for i in range(n)], np.int64)
    out_off = np.zeros(n + 1, np.int64)
    out_off[1:] = np.cumsum(caps)
    out = torch.empty(int(out_off[-1]), dtype=torch.uint8, device="cuda")
    out_off_d = torch.from_numpy(out_off).cuda()
    sizes = torch.empty(n, dtype=torch.int64, device="cuda")
    capi.check(L.pg_rans_encode_batch(symbols.data_ptr(), offsets.data_ptr(), n, out.data_ptr(),
                                      out_off_d.data_ptr(), sizes.data_ptr(), capi.stream_handle(stream)))
    return sizes


def store_sizes(slice_t, node_off, nodes, turn, stream=None):
    """The store coder on the same blocks (pg_store_*: rANS over a counted
    1024-context table of each rotation's neighbouring rotations and the
    previous node, no network): (stream bytes of each block, table bytes)."""
    import torch
    from .slice_store import store_bound
    L = capi.lib()
    sh = capi.stream_handle(stream)
    dev = slice_t.device
    k = len(node_off)
    t64 = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.int64)).to(dev)
    first = t64(node_off)
    count = torch.from_numpy(np.ascontiguousarray(nodes, dtype=np.int32)).to(dev)
    table = torch.empty(1024 * 3, dtype=torch.int16, device=dev)
    capi.check(L.pg_store_table(slice_t.data_ptr(), first.data_ptr(), count.data_ptr(), k, turn, table.data_ptr(), sh))
    caps = (store_bound(nodes) + 15) // 16 * 16
    out_off = np.zeros(k + 1, np.int64)
    out_off[1:] = np.cumsum(caps)
    out = torch.empty(int(out_off[-1]), dtype=torch.uint8, device=dev)
    sizes = torch.zeros(k, dtype=torch.int64, device=dev)
    capi.check(L.pg_store_encode(slice_t.data_ptr(), first.data_ptr(), count.data_ptr(), k, turn, table.data_ptr(),
                                 out.data_ptr(), t64(out_off[:-1]).data_ptr(), sizes.data_ptr(), sh))
    return sizes.cpu().numpy(), 2 * 1024 * 3


def run_slice_coding(root_counts=((4, 4), (4, 5), (4, 3), (3, 3)), train_fraction=0.01, steps=1500, batch=32768,
                chunk_blocks=4096, max_blocks=0, seed=1, sample_blocks=0, sweep_timings=None, sweep_counts=None):
    """Solve the root's sections down to its own slice, train on a
    seeded fraction of the root slice's blocks, code max_blocks blocks (0:
    all) both ways and check the round trip.  With sample_blocks > 0 the
    symbols of that many coded blocks are also returned on the host (for a
    CPU comparison); sweep_timings receives the sweep's per-slice timings and
    sweep_counts its per-slice section counts (as sweep.sweep returns them)."""
    import torch
    from . import sweep
    from .end import section_sig
    root = section_sig([list(c) for c in root_counts])
    slice_ = sum(sum(c) for c in root_counts)
    t0 = time.perf_counter()
    counts, slice_t, sigs = sweep.sweep(root, keep_last=True, timings=sweep_timings)
    if sweep_counts is not None:
        sweep_counts.update(counts)
    torch.cuda.synchronize()
    t_sweep = time.perf_counter() - t0
    layout = sweep.slice_layout(sigs)
    refs, node_off, nodes = slice_blocks(sigs, layout)
    nblocks = len(nodes) if not max_blocks else min(max_blocks, len(nodes))
    turn = slice_ & 1
    rng = np.random.default_rng(seed)
    ntrain = max(1, int(round(train_fraction * len(nodes))))
    tb = np.sort(rng.choice(len(nodes), ntrain, replace=False))
    trefs = subset(refs, tb)
    tsym, toff = block_symbols(slice_t, node_off[tb], nodes[tb], turn)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    tr = Trainer(trefs, tsym, toff, nodes[tb], seed=seed)
    hist = tr.run(steps, batch, log_every=max(1, steps // 10))
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    model = tr.model()
    del tsym, tr
    # Code the blocks spread evenly over the slice, chunk by chunk
    pick = np.unique(np.linspace(0, len(nodes) - 1, nblocks).astype(np.int64))
    tot = {"learned": 0, "static": 0, "store": 0, "symbols": 0, "enc_ms": 0.0, "dec_ms": 0.0, "static_streams": 0,
           "static_enc_ms": 0.0, "static_dec_ms": 0.0}
    lossless = True
    cpu_sample = None
    for c0 in range(0, len(pick), chunk_blocks):
        idx = pick[c0:c0 + chunk_blocks]
        crefs = subset(refs, idx)
        sym, off = block_symbols(slice_t, node_off[idx], nodes[idx], turn)
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        e0.record()
        data, doff, dsz = encode(model, crefs, sym, off, nodes[idx])
        e1.record()
        dec, _, status = decode(model, crefs, data, doff, dsz, nodes[idx])
        e2.record()
        torch.cuda.synchronize()
        tot["enc_ms"] += e0.elapsed_time(e1)
        tot["dec_ms"] += e1.elapsed_time(e2)
        ssz, s_enc, s_dec, s_ok = static_roundtrip(sym, off)
        tot["static_enc_ms"] += s_enc
        tot["static_dec_ms"] += s_dec
        lossless &= s_ok
        dsz_h = dsz.cpu().numpy()
        if (dsz_h < 0).any():
            raise RuntimeError("encode failed")
        tot["learned"] += int(dsz_h.sum())
        tot["static"] += int(ssz.sum().item())
        st_sz, st_table = store_sizes(slice_t, node_off[idx], nodes[idx], turn)
        tot["store"] += int(st_sz.sum()) + st_table
        tot["symbols"] += int(sym.numel())
        tot["static_streams"] += int((dsz_h == ssz.cpu().numpy()).sum())
        lossless &= bool(torch.equal(dec, sym)) and bool((status.cpu().numpy() == nodes[idx] * 256).all())
        if cpu_sample is None and sample_blocks > 0:
            k = min(sample_blocks, len(idx))
            o = off.cpu().numpy()
            cpu_sample = sym[:int(o[k])].cpu().numpy(), o[:k + 1]
        del sym, data, dec
    del slice_t
    torch.cuda.empty_cache()
    bits = lambda b: 8.0 * b / tot["symbols"]
    out = {
        "workload": f"all blocks of slice {slice_} below root {[list(c) for c in root_counts]} "
                    f"({'all' if len(pick) == len(nodes) else len(pick)} of {len(nodes)} blocks coded)",
        "blocks": int(len(pick)), "positions": tot["symbols"],
        "static_bits_per_position": bits(tot["static"]), "learned_bits_per_position": bits(tot["learned"]),
        "context_table_bits_per_position": bits(tot["store"]),
        "learned_over_static": tot["learned"] / tot["static"],
        "learned_over_context_table": tot["learned"] / tot["store"],
        "coders": {"static": "format 2: one order-0 table per block (the reference's coder)",
                   "context_table": "store coder: counted 1024-context table per chunk of blocks (the neighbouring "
                                    "rotations and the previous node's), table bytes included, no network",
                   "learned": "format 3: the MLP over the board, the rotation, the coded neighbouring rotations and "
                              "the previous node's symbol, model shared by the slice (not counted per block)"},
        "model_bytes": len(model),
        "blocks_kept_static": tot["static_streams"], "lossless": lossless,
        "encode_GBps_of_nodes": tot["symbols"] / 4 / (tot["enc_ms"] / 1e3) / 1e9,
        "decode_GBps_of_nodes": tot["symbols"] / 4 / (tot["dec_ms"] / 1e3) / 1e9,
        "encode_Msym_per_s": tot["symbols"] / (tot["enc_ms"] / 1e3) / 1e6,
        "decode_Msym_per_s": tot["symbols"] / (tot["dec_ms"] / 1e3) / 1e6,
        "static_gpu_encode_Msym_per_s": tot["symbols"] / (tot["static_enc_ms"] / 1e3) / 1e6,
        "static_gpu_decode_Msym_per_s": tot["symbols"] / (tot["static_dec_ms"] / 1e3) / 1e6,
        "train_blocks": int(ntrain), "train_steps": steps, "train_batch": batch, "train_s": t_train,
        "train_loss_bits": hist, "sweep_s": t_sweep}
    if sample_blocks > 0:
        return out, cpu_sample
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--root", default="4,4,4,5,4,3,3,3")
    ap.add_argument("--train-fraction", type=float, default=0.01)
    ap.add_argument("--steps", type=int, default=1500)
    ap.add_argument("--batch", type=int, default=32768)
    ap.add_argument("--chunk-blocks", type=int, default=4096)
    ap.add_argument("--max-blocks", type=int, default=0, help="code only N blocks spread over the slice (0: all)")
    ap.add_argument("--seed", type=int, default=1)
    args = ap.parse_args()
    c = [int(x) for x in args.root.split(",")]
    capi.check(capi.lib().pg_init())
    res = run_slice_coding(((c[0], c[1]), (c[2], c[3]), (c[4], c[5]), (c[6], c[7])), args.train_fraction, args.steps,
                      args.batch, args.chunk_blocks, args.max_blocks, args.seed)
    res["root"] = args.root
    print(json.dumps(res))


if __name__ == "__main__":
    main()
