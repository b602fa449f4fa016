"""End-engine kernels on the GPU, through the C ABI, against the oracle and the
reference's own outputs (golden SHA-1s made by oracle/_ref)."""
import ctypes

import numpy as np
import pytest

from tests.oracle import P
from tests.test_oracle import LINES, sha1, random_supers, random_sides

pytestmark = pytest.mark.gpu


def to_dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int64)).cuda()


def to_host(t):
    return t.cpu().numpy().view(np.uint64)


def test_device_superscore_matches_oracle(cuda, O):
    import torch
    from pentago_b200 import capi
    L = capi.lib()
    rng = np.random.default_rng(17)
    n = 1 << 16
    x = random_supers(rng, n)
    sides = random_sides(rng, n)
    syms = (np.arange(n) % 2048).astype(np.uint16)
    dx, ds = to_dev(x), to_dev(sides)
    dsym = torch.from_numpy(syms.view(np.int16)).cuda()
    dout = torch.zeros((n, 4), dtype=torch.int64, device=cuda)
    want = np.zeros_like(x)
    s = capi.stream_handle()
    for op, inp, oracle_fn, args in ((0, dx, O.rmax, (P(x),)), (1, ds, O.super_wins, (P(sides),)),
                                     (2, dx, O.transform_super, (P(syms), P(x)))):
        capi.check(L.pg_debug_super(op, inp.data_ptr(), dsym.data_ptr(), dout.data_ptr(), n, s))
        oracle_fn(*args, P(want), n)
        assert np.array_equal(to_host(dout), want), f"op {op}"


def gpu_line(case, flags=0, padded=False, prefill=None):
    import torch
    from pentago_b200 import end
    from pentago_b200.synthetic import random_nodes
    line = end.Line(case["section"], case["dimension"], case["block_base"], flags=flags)
    info = end.line_info(line)
    inp = random_nodes(case["seed"], max(info.input_nodes, 1))
    if padded:
        # The reference's own layout: one spare node after every child block
        # (end/compute.cc:84-94, :135-138).
        stride = info.block_stride + 1
        buf = np.full((info.input_blocks * stride, 8), 0xDEADBEEF, np.uint64)
        off = 0
        for k in range(info.input_blocks):
            nodes = min(info.block_stride, info.input_nodes - off)
            buf[k * stride:k * stride + nodes] = inp[off:off + nodes]
            off += nodes
        line.input_block_stride = stride
        inp = buf
    line.input = to_dev(inp)
    out = np.zeros((info.output_nodes, 8), np.uint64) if prefill is None else prefill
    line.output = to_dev(out)
    end.compute_lines([line])
    end.check_errors()
    return to_host(line.output)


@pytest.mark.parametrize("case", LINES, ids=lambda c: f"{c['counts']}-{c['dimension']}")
def test_line_kernel_matches_reference_golden(cuda, case):
    assert sha1(gpu_line(case)) == case["output_sha1"]


@pytest.mark.parametrize("case", LINES[:3], ids=lambda c: f"{c['counts']}-{c['dimension']}")
def test_line_kernel_reference_padded_layout_and_or_mode(cuda, case):
    base = gpu_line(case)
    assert sha1(gpu_line(case, padded=True)) == case["output_sha1"]
    from pentago_b200.synthetic import random_nodes
    prior = random_nodes(99, base.shape[0])
    got = gpu_line(case, flags=1, prefill=prior.copy())
    assert np.array_equal(got, base | prior)


def test_single_block_30_stone_section_matches_oracle(cuda, O):
    """One 8^4 block of the 30-stone section [[4,4],[4,4],[4,3],[3,4]]: the OR
    of the four block lines through block (1,1,1,1), on seeded children."""
    import torch
    from pentago_b200 import end
    from pentago_b200.synthetic import random_nodes
    sig = end.section_sig([[4, 4], [4, 4], [4, 3], [3, 4]])
    block = (1, 1, 1, 1)
    got = None
    want = None
    for dim in range(4):
        bb = tuple(block[i] for i in range(4) if i != dim)
        line = end.Line(sig, dim, bb)
        info = end.line_info(line)
        inp = random_nodes(1 + dim, info.input_nodes)
        line.input = to_dev(inp)
        line.output = torch.zeros((info.output_nodes, 8), dtype=torch.int64, device=cuda)
        end.compute_lines([line])
        ref = np.zeros((info.output_nodes, 8), np.uint64)
        O.compute_line(sig, dim, line.length, (ctypes.c_uint8 * 3)(*bb), P(inp), P(ref), 8)
        # The block is block index `block[dim]` along the line
        s = info.block_stride
        g = to_host(line.output)[block[dim] * s:(block[dim] + 1) * s]
        w = ref[block[dim] * s:(block[dim] + 1) * s]
        # Lines store blocks in the line's axis order; reorder to the block's row-major order
        shape = list(info.output_shape)
        shape[dim] = 8
        perm_shape = shape
        g = g.reshape(perm_shape + [8])
        w = w.reshape(perm_shape + [8])
        got = g if got is None else got | g
        want = w if want is None else want | w
    end.check_errors()
    assert np.array_equal(got, want)
    assert got.any()


def test_prepared_plan_runs_repeatedly(cuda):
    """pg_end_plan_create / run / destroy: the same lines run twice give the golden output."""
    import torch
    from pentago_b200 import end
    from pentago_b200.synthetic import random_nodes
    lines, want = [], []
    for case in LINES[:5]:
        line = end.Line(case["section"], case["dimension"], case["block_base"])
        info = end.line_info(line)
        line.input = to_dev(random_nodes(case["seed"], max(info.input_nodes, 1)))
        line.output = torch.zeros((info.output_nodes, 8), dtype=torch.int64, device=cuda)
        lines.append(line)
        want.append(case["output_sha1"])
    plan = end.Plan(lines)
    assert plan.streams == 4   # four dimensions, every line its own output
    for _ in range(2):
        for l in lines:
            l.output.zero_()
        plan.run()
        end.check_errors()
        assert [sha1(to_host(l.output)) for l in lines] == want
    plan.close()


def test_plan_streams_follow_line_independence(cuda):
    """The four lines through one block of a 30-stone section, writing
    disjoint parts of one buffer, run on four streams and give what one call
    per line gives; lines that OR into their outputs, or whose outputs
    overlap, run on one stream."""
    import torch
    from pentago_b200 import capi, end
    from pentago_b200.synthetic import random_nodes
    sig = end.section_sig([[4, 4], [4, 4], [4, 3], [3, 4]])
    lines, infos = [], []
    for dim in range(4):
        line = end.Line(sig, dim, (0, 0, 0))
        info = end.line_info(line)
        line.input = to_dev(random_nodes(10 + dim, info.input_nodes))
        lines.append(line)
        infos.append(info)
    total = sum(i.output_nodes for i in infos)
    shared = torch.full((total, 8), -1, dtype=torch.int64, device=cuda)
    o = 0
    for line, info in zip(lines, infos):
        line.output = shared[o:o + info.output_nodes]
        o += info.output_nodes
    plan = end.Plan(lines)
    assert plan.streams == 4
    plan.run()
    end.check_errors()
    got = shared.clone()
    o = 0
    for line, info in zip(lines, infos):
        alone = torch.zeros((info.output_nodes, 8), dtype=torch.int64, device=cuda)
        single = end.Line(sig, line.dimension, line.block_base)
        single.input, single.output = line.input, alone
        end.compute_lines([single])
        assert torch.equal(got[o:o + info.output_nodes], alone), line.dimension
        o += info.output_nodes
    plan.close()
    # OR into the outputs: one stream
    for line in lines:
        line.flags = capi.PG_LINE_OR
    assert end.Plan(lines).streams == 1
    # outputs of two dimensions that overlap: one stream
    for line in lines:
        line.flags = capi.PG_LINE_STORE
    lines[1].output = shared[8:8 + infos[1].output_nodes]
    assert end.Plan(lines).streams == 1
    # one dimension only: one stream
    assert end.Plan(lines[:1]).streams == 1
