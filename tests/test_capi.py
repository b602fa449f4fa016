"""The C-ABI library: it loads, exports every symbol include/pentago_b200.h
declares, builds tables identical to the reference generator's, and its kernel
arithmetic (run on the host) matches the oracle.  No GPU."""
import ctypes
import hashlib
import json
import os
import re

import numpy as np
import pytest

from tests.oracle import P
from tests.test_oracle import HASHES, TABLES, LINES, sha1, random_supers, random_sides

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    text = open(os.path.join(ROOT, "include", "pentago_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(pg_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    from pentago_b200 import capi
    lib = capi.lib()
    names = header_functions()
    assert len(names) >= 10
    for n in names:
        assert hasattr(lib, n), n
        assert n in capi.SIGNATURES, f"{n} has no ctypes signature"


@pytest.mark.parametrize("name,dtype,key,idx,cast", TABLES)
def test_product_tables_match_precompute_sha1(name, dtype, key, idx, cast):
    from pentago_b200 import capi
    n = ctypes.c_int()
    p = capi.lib().pg_selftest_table(name.encode(), ctypes.byref(n))
    t = np.frombuffer((ctypes.c_char * n.value).from_address(p), dtype=dtype).copy()
    if cast:
        t = t.astype(np.uint64)
    assert sha1(t) == HASHES[key][idx]


def test_kernel_superscore_on_host_matches_oracle(O):
    from pentago_b200 import capi
    L = capi.lib()
    rng = np.random.default_rng(3)
    n = 4096
    x = random_supers(rng, n)
    a, b = np.zeros_like(x), np.zeros_like(x)
    capi.check(L.pg_selftest_super_host(0, P(x), None, P(a), n))
    O.rmax(P(x), P(b), n)
    assert np.array_equal(a, b)
    sides = random_sides(rng, n)
    capi.check(L.pg_selftest_super_host(1, P(sides), None, P(a), n))
    O.super_wins(P(sides), P(b), n)
    assert np.array_equal(a, b)
    syms = (np.arange(n) % 2048).astype(np.uint16)
    capi.check(L.pg_selftest_super_host(2, P(x), P(syms), P(a), n))
    O.transform_super(P(syms), P(x), P(b), n)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("case", LINES, ids=lambda c: f"{c['counts']}-{c['dimension']}")
def test_kernel_line_code_on_host_matches_reference_golden(case):
    from pentago_b200 import end
    from pentago_b200.synthetic import random_nodes
    line = end.Line(case["section"], case["dimension"], case["block_base"])
    info = end.line_info(line)
    assert (info.input_nodes, info.output_nodes) == (case["input_nodes"], case["output_nodes"])
    line.input = random_nodes(case["seed"], max(case["input_nodes"], 1))
    line.output = np.zeros((case["output_nodes"], 8), np.uint64)
    end.selftest_lines_host([line])
    assert sha1(line.output) == case["output_sha1"]


def random_section(rng, stones):
    """A valid section with `stones` stones (black has the extra one when odd)."""
    c = [[0, 0] for _ in range(4)]
    for color, cnt in ((0, (stones + 1) // 2), (1, stones // 2)):
        for _ in range(cnt):
            free = [q for q in range(4) if sum(c[q]) < 9]
            c[free[int(rng.integers(len(free)))]][color] += 1
    return c


def test_kernel_line_code_on_host_matches_oracle_for_every_symmetry(O):
    """Random block lines of 33- to 35-stone sections, run through the
    kernel's own microline code on the host, equal the oracle's line compute;
    between them the lines' children are standardized by each of the 8 global
    symmetries (the per-line axis maps of the children's transform)."""
    import collections
    from pentago_b200 import end
    from pentago_b200.synthetic import random_nodes
    rng = np.random.default_rng(123)
    seen = collections.Counter()
    n = 0
    while n < 60:
        stones = int(rng.integers(33, 36))
        c = random_section(rng, stones)
        dims = [d for d in range(4) if sum(c[d]) < 9]
        if not dims:
            continue
        dim = dims[int(rng.integers(len(dims)))]
        sig = end.section_sig(c)
        shape = end.section_shape(sig)
        bb = tuple(int(rng.integers((shape[i] + 7) // 8)) for i in range(4) if i != dim)
        line = end.Line(sig, dim, bb)
        info = end.line_info(line)
        if info.output_nodes > 40000:
            continue
        inp = random_nodes(n + 7, max(info.input_nodes, 1))
        got = np.zeros((info.output_nodes, 8), np.uint64)
        want = np.zeros_like(got)
        line.input, line.output = inp, got
        end.selftest_lines_host([line])
        O.compute_line(sig, dim, line.length, (ctypes.c_uint8 * 3)(*bb), P(inp), P(want), 8)
        assert np.array_equal(got, want), (c, dim, bb)
        child = [[c[q][k] + (q == dim and k == stones % 2) for k in range(2)] for q in range(4)]
        seen[end.section_standardize(end.section_sig(child))[1]] += 1
        n += 1
    assert sorted(seen) == list(range(8)), seen


def test_line_rejects_bad_input():
    from pentago_b200 import capi, end
    full = end.section_sig([[5, 4], [4, 5], [4, 4], [4, 3]])
    with pytest.raises(capi.PentagoError):
        end.line_info(end.Line(full, 0, (0, 0, 0), length=5))   # quadrant 0 is full
    with pytest.raises(capi.PentagoError):
        end.line_info(end.Line(end.section_sig([[4, 4], [4, 4], [4, 3], [3, 4]]), 0, (0, 0, 0), length=3))
    with pytest.raises(capi.PentagoError):
        end.line_info(end.Line(end.section_sig([[1, 4], [4, 4], [4, 3], [3, 4]]), 0, (0, 0, 0), length=1))


def test_sweep_child_refuses_unstandardized_sections():
    from pentago_b200 import capi
    from pentago_b200.end import section_sig
    L = capi.lib()
    sig = section_sig([[4, 4], [4, 5], [4, 3], [3, 3]])
    parents = np.array([sig], np.uint64)
    bad = section_sig([[3, 3], [4, 3], [4, 5], [4, 4]])   # not standardized
    dummy = np.zeros(8, np.uint64)
    assert L.pg_end_sweep_slice_child(P(parents), 1, P(dummy), bad, P(dummy), None) == capi.PG_ERR_ARG


def test_deep_root_slices_and_golden_rows():
    """The 28-stone root of the compressed-sweep test: its two largest
    adjacent slices need more than a B200 holds raw, and the committed golden
    rows cover exactly its sections at slices 28 and 29."""
    from pentago_b200 import sweep
    from pentago_b200.end import section_sig
    from tests.test_slice_store_gpu import DEEP_ROOT
    root = section_sig(DEEP_ROOT)
    nodes = {s: int(sweep.slice_layout(sweep.descendent_sections(root, s))[-1]) for s in range(28, 36)}
    assert 64 * max(nodes[s] + nodes[s + 1] for s in range(28, 35)) > 192e9
    gold = np.load(os.path.join(os.path.dirname(__file__), "golden", "counts_28_29.npz"))
    for s in (28, 29):
        assert sorted(int(r[0]) for r in gold[f"counts_{s}"]) == [int(x) for x in sweep.descendent_sections(root, s)]


def test_store_bound_matches_the_library():
    """slice_store.store_bound (what compressed_slice reserves per block) is
    the library's pg_store_bound for every block size up to a full block."""
    from pentago_b200 import capi
    from pentago_b200.slice_store import store_bound
    L = capi.lib()
    counts = np.arange(0, 4097)
    assert store_bound(counts).tolist() == [L.pg_store_bound(int(c)) for c in counts]
    assert L.pg_store_bound(-1) == capi.PG_ERR_ARG


def test_sweep_arena_halves_hold_every_adjacent_pair():
    """The raw sweep's two arena halves (slices alternate between them) add
    up to the largest pair of adjacent slices for the root [[4,4],[4,5],[4,3],[3,3]], whose
    slice sizes rise and then fall: 63.5 + 78.2 = 141.7 GB."""
    from pentago_b200 import sweep
    from pentago_b200.end import section_sig
    root = section_sig([[4, 4], [4, 5], [4, 3], [3, 3]])
    chain = list(range(35, 29, -1))
    halves = sweep._arena_nodes(root, chain)
    nodes = [int(sweep.slice_layout(sweep.descendent_sections(root, s))[-1]) for s in chain]
    assert sum(halves) == max(a + b for a, b in zip(nodes, nodes[1:]))
    assert round(64 * sum(halves) / 1e9, 1) == 141.7
    # every slice fits the half it is placed in
    assert all(n <= halves[k % 2] for k, n in enumerate(nodes))


def all_sections(slice_):
    """Every standardized section of a slice (all_boards_sections(slice, 8),
    pentago/base/all_boards.cc): each split of the stones over the quadrants,
    through pg_section_standardize, without duplicates."""
    from pentago_b200 import capi
    from pentago_b200.end import section_sig
    L = capi.lib()
    std, tr = ctypes.c_uint64(), ctypes.c_int32()
    pairs = [(b, w) for b in range(10) for w in range(10) if b + w <= 9]
    seen = set()

    def rec(cs, black, white):
        if len(cs) == 3:
            if black + white <= 9:
                capi.check(L.pg_section_standardize(ctypes.c_uint64(section_sig(cs + [[black, white]])),
                                                    ctypes.byref(std), ctypes.byref(tr)))
                seen.add(int(std.value))
            return
        for b, w in pairs:
            if b <= black and w <= white:
                rec(cs + [[b, w]], black - b, white - w)
    rec([], (slice_ + 1) // 2, slice_ // 2)
    return np.array(sorted(seen), np.uint64)


def test_slice_totals_match_end_test():
    """The nodes, 8^4 blocks and block lines (dimensions whose quadrant is
    not full) of every 24-stone section, from the library's section algebra
    and shapes, equal the totals in pentago/end/end_test.cc."""
    from pentago_b200 import sweep
    from pentago_b200.end import section_shape
    gold = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "end_totals.json")))
    sigs = all_sections(gold["slice"])
    blocks = lines = 0
    for s in sigs:
        nb = (np.array(section_shape(int(s))) + 7) // 8
        blocks += int(np.prod(nb))
        counts = [[(int(s) >> (16 * q + 8 * k)) & 255 for k in range(2)] for q in range(4)]
        lines += sum(int(np.prod(np.delete(nb, d))) for d in range(4) if sum(counts[d]) < 9)
    assert int(sweep.slice_layout(sigs)[-1]) == gold["nodes"]
    assert blocks == gold["blocks"] and lines == gold["lines"]


def test_block_enumerations_agree_and_tile_the_slice():
    """The three host enumerations of a slice's 8^4 blocks (slice files,
    compressed slices, the learned coder) give the same node offsets and
    counts, and the blocks tile the slice tensor exactly, on a slice with
    ragged sections."""
    from pentago_b200 import learned, slice_store, supertensor, sweep
    from pentago_b200.end import section_sig
    sigs = sweep.descendent_sections(section_sig([[4, 4], [4, 5], [4, 3], [3, 3]]), 33)
    layout = sweep.slice_layout(sigs)
    _, first, count, _, _ = slice_store.slice_blocks(sigs)
    _, _, offs, total = supertensor._slice_blocks(sigs)
    _, loffs, lcount = learned.slice_blocks(sigs, layout)
    assert np.array_equal(first, offs) and np.array_equal(first, loffs)
    assert np.array_equal(count, lcount)
    assert total == int(layout[-1]) == int(count.sum())
    assert first[0] == 0 and np.array_equal(first[1:], first[:-1] + count[:-1])
    assert (count < 4096).any() and (count == 4096).any()
