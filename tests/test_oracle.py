"""The CPU oracle pinned against the reference's golden vectors and the
reference engine itself (oracle/_ref).  No GPU."""
import ctypes
import hashlib
import json
import os

import numpy as np
import pytest

from tests.oracle import P

GOLD = os.path.join(os.path.dirname(__file__), "golden")
HASHES = json.load(open(os.path.join(GOLD, "tables_sha1.json")))


def sha1(a):
    return hashlib.sha1(np.ascontiguousarray(a).tobytes()).hexdigest()


# (table name, dtype, golden key, index in that key's list, cast to uint64 first)
TABLES = [("pack_table", np.uint16, "pack", 0, False),
          ("unpack_table", np.uint16, "unpack", 0, False),
          ("rotations", np.uint16, "table", 1, False),
          ("reflections", np.uint16, "table", 5, False),
          ("commute_global_local_symmetries", np.uint8, "table", 6, True),
          ("rotation_minimal_quadrants_offsets", np.uint16, "nest.offsets", 0, True),
          ("rotation_minimal_quadrants_flat", np.uint16, "nest.flat", 0, True),
          ("rotation_minimal_quadrants_inverse", np.uint16, "inverse", 0, True),
          ("rotation_minimal_quadrants_reflect_moved", np.uint16, "moved", 0, True)]


@pytest.mark.parametrize("name,dtype,key,idx,cast", TABLES)
def test_oracle_tables_match_precompute_sha1(O, name, dtype, key, idx, cast):
    t = O.get_table(name, dtype)
    if cast:
        t = t.astype(np.uint64)
    assert sha1(t) == HASHES[key][idx]


def random_supers(rng, n):
    return rng.integers(0, 2**64, size=(n, 4), dtype=np.uint64)


def random_sides(rng, n):
    q = rng.integers(0, 512, size=(n, 4)) & rng.integers(0, 512, size=(n, 4)) | \
        rng.integers(0, 512, size=(n, 4)) & rng.integers(0, 512, size=(n, 4))
    return (q[:, 0] | q[:, 1] << 16 | q[:, 2] << 32 | q[:, 3] << 48).astype(np.uint64)


def test_oracle_superscore_vs_reference(O, R):
    rng = np.random.default_rng(11)
    n = 4000
    x = random_supers(rng, n)
    for f in ("rmax",):
        a, b = np.zeros_like(x), np.zeros_like(x)
        getattr(O, f)(P(x), P(a), n)
        getattr(R, f)(P(x), P(b), n)
        assert np.array_equal(a, b), f
    sides = random_sides(rng, n)
    a, b = np.zeros_like(x), np.zeros_like(x)
    O.super_wins(P(sides), P(a), n)
    R.super_wins(P(sides), P(b), n)
    assert np.array_equal(a, b) and a.any()
    syms = np.arange(n, dtype=np.uint16) % 2048  # every symmetry
    O.transform_super(P(syms), P(x), P(a), n)
    R.transform_super(P(syms), P(x), P(b), n)
    assert np.array_equal(a, b)
    s2 = rng.integers(0, 2048, size=n).astype(np.uint16)
    pa, pb = np.zeros(n, np.uint16), np.zeros(n, np.uint16)
    O.symmetry_product(P(syms), P(s2), P(pa), n)
    R.symmetry_product(P(syms), P(s2), P(pb), n)
    assert np.array_equal(pa, pb)
    par = rng.integers(0, 2, size=n).astype(np.uint8)
    ha, hb = np.zeros((n, 2), np.uint64), np.zeros((n, 2), np.uint64)
    O.halfsuper_wins(P(sides), P(par), P(ha), n)
    R.halfsuper_wins(P(sides), P(par), P(hb), n)
    assert np.array_equal(ha, hb)
    hx = x[:, :2].copy()
    O.halfsuper_rmax(P(hx), P(ha), n)
    R.halfsuper_rmax(P(hx), P(hb), n)
    assert np.array_equal(ha, hb)


LINES = json.load(open(os.path.join(GOLD, "lines.json")))


def run_oracle_line(O, case):
    from pentago_b200.synthetic import random_nodes
    inp = random_nodes(case["seed"], max(case["input_nodes"], 1))
    out = np.zeros((case["output_nodes"], 8), np.uint64)
    bb = (ctypes.c_uint8 * 3)(*case["block_base"])
    O.compute_line(case["section"], case["dimension"], case["length"], bb, P(inp), P(out), os.cpu_count() or 1)
    return out


@pytest.mark.parametrize("case", LINES[:4], ids=lambda c: f"{c['counts']}-{c['dimension']}")
def test_oracle_lines_match_reference_golden(O, case):
    assert sha1(run_oracle_line(O, case)) == case["output_sha1"]


def test_oracle_workspace_sizes(O):
    w = json.load(open(os.path.join(GOLD, "workspace.json")))
    for i, size in enumerate(w["sizes"]):
        assert O.midsolve_workspace_size(w["first_slice"] + i) == size


def board_from_cells(cells):
    q = [0] * 4
    for qx in range(2):
        for qy in range(2):
            v = 0
            for i in range(9):
                x, y = i // 3, i % 3
                c = cells[(3 * qx + x) * 6 + 3 * qy + y]
                v += 3 ** i * c
            q[2 * qx + qy] = v
    return q[0] | q[1] << 16 | q[2] << 32 | q[3] << 48


def test_oracle_midsolve_vs_reference(O, R):
    rng = np.random.default_rng(5)
    for stones in (34, 32, 30, 28, 27, 26):
        for _ in range(4):
            cells = [0] * 36
            perm = rng.permutation(36)
            for i in range(stones):
                cells[perm[i]] = 1 if i < (stones + 1) // 2 else 2
            b = board_from_cells(cells)
            for middle in (0, 1):
                raw = b | middle << 63
                ra, va = np.zeros(200, np.uint64), np.zeros(200, np.int32)
                rb, vb = np.zeros(200, np.uint64), np.zeros(200, np.int32)
                na = O.midsolve(raw, P(ra), P(va))
                nb = R.midsolve(raw, P(rb), P(vb))
                assert na == nb and np.array_equal(ra[:na], rb[:na]) and np.array_equal(va[:na], vb[:na])


def test_reference_build_matches_golden_midsolve_18(R):
    g = json.load(open(os.path.join(GOLD, "midsolve_18.json")))
    raws, vals = np.zeros(200, np.uint64), np.zeros(200, np.int32)
    n = R.midsolve(g["root"], P(raws), P(vals))
    want = {(b | m << 63): v for b, m, v in g["results"]}
    assert n == len(want) == 163
    assert {int(r): int(v) for r, v in zip(raws[:n], vals[:n])} == want
