"""Slice files on the GPU: the filter kernels against the oracle, the device
write path against the reference's supertensor test hash, the reference's
solved database read into a slice tensor and counted on the GPU against
data/counts-N.npy, and a sweep that checkpoints every slice and resumes from
one of them with the same results."""
import hashlib
import os

import numpy as np
import pytest

from tests.oracle import P
from tests.test_supertensor_cpu import GOLDEN, ST, reference_blocks

pytestmark = pytest.mark.gpu


def random_nodes(n, seed):
    rng = np.random.default_rng(seed)
    win = rng.integers(0, 2**64 - 1, size=(n, 4), dtype=np.uint64, endpoint=True)
    nl = win | rng.integers(0, 2**64 - 1, size=(n, 4), dtype=np.uint64, endpoint=True)
    return np.ascontiguousarray(np.concatenate([win, nl], 1))


def test_filter_kernels_match_oracle(cuda, O):
    import torch
    from pentago_b200 import capi
    L = capi.lib()
    for n in (1, 7, 4096, 100003):
        nodes = random_nodes(n, n)
        dev = torch.from_numpy(nodes.view(np.int64)).cuda()
        for turn in (0, 1, 2):
            for filt in (0, 1):
                out = torch.empty_like(dev)
                capi.check(L.pg_supertensor_filter(dev.data_ptr(), n, turn, filt, out.data_ptr(), None))
                want = np.zeros_like(nodes)
                O.st_filter(P(nodes), n, turn, filt, P(want))
                assert np.array_equal(out.cpu().numpy().view(np.uint64), want), (n, turn, filt)
                back = torch.empty_like(dev)
                capi.check(L.pg_supertensor_unfilter(out.data_ptr(), n, turn, filt, back.data_ptr(), None))
                assert torch.equal(back, dev), (n, turn, filt)


def test_device_writer_matches_reference_hash(cuda, tmp_path):
    import torch
    from pentago_b200 import supertensor
    sig, h, data = reference_blocks()
    path = str(tmp_path / "test.pentago")
    w = supertensor.supertensor_writer_t(path, sig, ST["block_size"], ST["filter"], ST["level"])
    for b in ST["write_order"]:
        w.write_block(b, torch.from_numpy(data[tuple(b)].view(np.int64)).cuda(), turn=supertensor.RAW)
    w.finalize()
    w.close()
    assert hashlib.sha1(open(path, "rb").read()).hexdigest() in ST["sha1"]
    r = supertensor.supertensor_reader_t(path)
    for b in np.ndindex(*ST["blocks"]):
        got = r.read_block(b, turn=supertensor.RAW)
        assert tuple(got.shape[:4]) == h.block_shape(b)
        assert np.array_equal(got.reshape(-1, 8).cpu().numpy().view(np.uint64), data[b])
    # many blocks in one call, into one tensor at scattered offsets
    blocks = [tuple(b) for b in np.ndindex(*ST["blocks"])][::-1]
    sizes = [len(data[b]) for b in blocks]
    offs = np.concatenate([[0], np.cumsum(sizes)[:-1]]) + 3
    out = torch.zeros((sum(sizes) + 3, 8), dtype=torch.int64, device="cuda")
    r.read_blocks(blocks, out, offs)
    host = out.cpu().numpy().view(np.uint64)
    assert not host[:3].any()
    for b, o in zip(blocks, offs):
        assert np.array_equal(host[o:o + len(data[b])], data[b])


def test_database_counts_on_gpu(cuda):
    """The reference's solved slices 0..5 read into slice tensors (GPU
    unfilter) and counted by the GPU count kernel give data/counts-N.npy."""
    import torch
    from pentago_b200 import capi, supertensor
    from pentago_b200.sweep import to_golden
    gold = np.load(os.path.join(GOLDEN, "counts_0_5.npz"))
    for s in range(6):
        slice_, sigs, nodes = supertensor.read_slice(os.path.join(GOLDEN, "db", f"slice-{s}.pentago"))
        assert slice_ == s
        counts = torch.zeros((len(sigs), 3), dtype=torch.int64, device="cuda")
        capi.check(capi.lib().pg_section_counts(capi.ptr(sigs), len(sigs), nodes.data_ptr(), counts.data_ptr(), None))
        rows = to_golden(sigs, counts.cpu().numpy().view(np.uint64), s)
        want = {int(r[0]): r for r in gold[f"counts_{s}"]}
        assert len(rows) == len(want)
        for r in rows:
            assert np.array_equal(r, want[int(r[0])]), (s, r)


def test_sweep_checkpoint_and_resume(cuda, tmp_path):
    """A 33-stone root solved with a checkpoint per slice; the files read back
    equal the slice tensors, and resuming from slice 34 gives slice 33 again."""
    import torch
    from pentago_b200 import supertensor, sweep
    from pentago_b200.end import section_sig
    root = section_sig([[4, 4], [5, 4], [4, 5], [4, 3]])
    res, last, sigs = sweep.sweep(root, keep_last=True, checkpoint=str(tmp_path), level=1)
    assert sorted(res) == [33, 34, 35]
    for s in (35, 34, 33):
        assert supertensor.supertensor_slice(str(tmp_path / f"slice-{s}.pentago")) == s
    slice_, sigs2, back = supertensor.read_slice(str(tmp_path / "slice-33.pentago"))
    assert slice_ == 33 and np.array_equal(sigs2, sigs)
    assert torch.equal(back, last)
    del back
    res2 = sweep.sweep(root, resume=str(tmp_path / "slice-34.pentago"))
    assert sorted(res2) == [33]
    assert np.array_equal(res2[33], res[33])
