"""Generate the golden fixtures in tests/golden/ from the reference repository.

Run in a container that has the reference sources and the in-place reference
build (``make -C oracle ref``):

    python tests/golden/make_golden.py /path/to/pentago

Fixtures written:
  tables_sha1.json   SHA-1 hashes embedded in pentago/base/precompute.cc's check() calls
  midsolve_18.json   the 18-stone board and its 163 (board, middle, value) results from
                     pentago/mid/benchmark_test.cc (read from the test source)
  high_samples.json  the (board, wins[8]) samples of pentago/high/high_test.cc:41-85
  workspace.json     midsolve workspace sizes of pentago/mid/mid_test.cc:129-134
  counts_30_35.npz   per-section (sig, black wins, white wins, total) rows from
                     data/counts-{30..35}.npy
  lines.json         block lines computed by the reference engine itself (oracle/_ref)
                     on seeded inputs: the seed and the SHA-1 of the output
  supertensor.json   the parameters and expected file SHA-1s of
                     pentago/data/supertensor_test.cc, with the order in which that
                     test writes its blocks (its unordered_map's iteration order,
                     taken from the reference compiled in place)
  db/slice-N.pentago the reference's solved database for slices 0..5 (data/), its
                     index files (slice-N.pentago.index), the sizes of the index
                     files of slices 6..8 (index_sizes.json), and
  counts_0_5.npz     its per-section counts (data/counts-{0..5}.npy)
  shards.json        pentago/shard/sharder_test.cc's server-verified (board, value)
                     samples of shard 7 of 32 over slices 0..5, and the per-slice
                     entry counts listed in pentago/shard/shard_permute.h
  counts_28_29.npz   the rows of data/counts-{28,29}.npy for the sections of the
                     28-stone root DEEP_ROOT at slices 28 and 29 (with
                     counts_30_35.npz, every section of its sweep)
  end_totals.json    the node, block and line totals of every 24-stone section
                     in pentago/end/end_test.cc (TEST(end, simple_partition))
"""
import ctypes
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))


# Lines covering: rotation-only and reflected child sections, every dimension,
# a 35-stone section (no children), duplicate-quadrant sections, short last blocks.
LINE_CASES = [([[4, 4], [4, 5], [4, 3], [4, 4]], 2, (1, 0, 1)),
              ([[3, 5], [5, 3], [4, 4], [5, 4]], 1, (0, 1, 0)),
              ([[4, 5], [4, 4], [5, 4], [4, 3]], 3, (0, 0, 0)),
              ([[5, 4], [4, 5], [4, 4], [4, 4]], 2, (0, 0, 1)),
              ([[4, 4], [5, 4], [4, 4], [4, 4]], 0, (1, 2, 2)),
              ([[5, 4], [4, 5], [4, 4], [4, 4]], 3, (0, 0, 0)),
              ([[5, 4], [4, 4], [4, 5], [4, 4]], 1, (0, 0, 0)),
              ([[5, 4], [4, 5], [5, 4], [4, 4]], 3, (0, 0, 0)),
              ([[4, 4], [4, 4], [4, 3], [3, 4]], 0, (1, 1, 1)),
              ([[4, 4], [4, 4], [4, 3], [3, 4]], 3, (1, 1, 1))]


# A 28-stone root whose two largest adjacent slices (31 and 30: 105.4 + 99.5 GB)
# do not fit a B200's HBM raw; its sweep needs slices kept compressed.
DEEP_ROOT = [[4, 4], [4, 5], [4, 3], [2, 2]]


def deep_root_counts(ref_root):
    from pentago_b200.end import section_sig
    from pentago_b200.sweep import descendent_sections
    out = {}
    for s in (28, 29):
        want = {int(x) for x in descendent_sections(section_sig(DEEP_ROOT), s)}
        rows = np.load(os.path.join(ref_root, "data", f"counts-{s}.npy"))
        rows = rows[[int(r[0]) in want for r in rows]]
        assert len(rows) == len(want)
        out[f"counts_{s}"] = rows
    np.savez_compressed(os.path.join(HERE, "counts_28_29.npz"), **out)


def numbers(text):
    return [int(x) for x in re.findall(r"-?\d+", text)]


def main(ref_root):
    src = lambda p: open(os.path.join(ref_root, p)).read()
    # 1. table hashes
    pre = src("pentago/base/precompute.cc")
    hashes = {}
    for m in re.finditer(r'check(?:<uint64_t>)?\((\w+(?:\.\w+)?), "([0-9a-f]{40})"\)', pre):
        hashes.setdefault(m.group(1), []).append(m.group(2))
    json.dump(hashes, open(os.path.join(HERE, "tables_sha1.json"), "w"), indent=1)

    # 2. midsolve golden (benchmark_test.cc)
    bt = src("pentago/mid/benchmark_test.cc")
    raw0 = re.search(r"raw0 = \{(.*?)\};", bt, re.S).group(1)
    raw1 = re.search(r"raw1 = \{(.*?)\};", bt, re.S).group(1)
    pairs0 = [(b, v) for b, v in re.findall(r"\{(\d+),(-?\d+)\}", raw0)]
    pairs1 = [(b, v) for b, v in re.findall(r"\{(\d+),(-?\d+)\}", raw1)]
    root = int(re.search(r"from_board\((\d+), false\);\n\s+const auto results", bt).group(1))
    json.dump({"root": root,
               "results": [[int(b), 0, int(v)] for b, v in pairs0] + [[int(b), 1, int(v)] for b, v in pairs1]},
              open(os.path.join(HERE, "midsolve_18.json"), "w"))

    # 3. high_test samples
    ht = src("pentago/high/high_test.cc")
    samples = {}
    for m in re.finditer(r"TEST\(high, board_(\d+)\) \{\s*const board_t boards\[\] = \{(.*?)\};\s*"
                         r"const uint64_t wins\[\] = \{(.*?)\};", ht, re.S):
        samples[m.group(1)] = {"boards": [int(x) for x in re.findall(r"\d+", m.group(2))],
                               "wins": [int(x) for x in re.findall(r"\d+", m.group(3))]}
    json.dump(samples, open(os.path.join(HERE, "high_samples.json"), "w"))

    # 4. workspace sizes
    mt = src("pentago/mid/mid_test.cc")
    ws = numbers(re.search(r"const int correct\[\] = \{(.*?)\};", mt, re.S).group(1))
    json.dump({"first_slice": 18, "sizes": ws}, open(os.path.join(HERE, "workspace.json"), "w"))

    # 5. golden section counts
    counts = {}
    for s in range(30, 36):
        counts[f"counts_{s}"] = np.load(os.path.join(ref_root, "data", f"counts-{s}.npy"))
    np.savez_compressed(os.path.join(HERE, "counts_30_35.npz"), **counts)

    # 6. reference-computed lines: inputs are regenerated from the seed, only
    #    the SHA-1 of the reference engine's output is stored
    import hashlib
    from tests.oracle import reference, P
    from pentago_b200.end import section_sig, section_shape
    from pentago_b200.synthetic import random_nodes
    R = reference()
    assert R is not None, "build oracle/_ref first (make -C oracle ref)"
    lines = []
    for k, (c, dim, bb) in enumerate(LINE_CASES):
        sig = section_sig(c)
        length = (section_shape(sig)[dim] + 7) // 8
        ni, no = ctypes.c_int64(), ctypes.c_int64()
        bbv = (ctypes.c_uint8 * 3)(*bb)
        R.line_sizes(sig, dim, length, bbv, ctypes.byref(ni), ctypes.byref(no))
        seed = 1000 + k
        inp = random_nodes(seed, max(ni.value, 1))
        res = np.zeros((no.value, 8), np.uint64)
        R.compute_line(sig, dim, length, bbv, P(inp), P(res), 0)
        lines.append({"counts": c, "section": sig, "dimension": dim, "block_base": list(bb), "length": length,
                      "seed": seed, "input_nodes": ni.value, "output_nodes": no.value,
                      "output_sha1": hashlib.sha1(res.tobytes()).hexdigest()})
    json.dump(lines, open(os.path.join(HERE, "lines.json"), "w"), indent=1)

    # 7. supertensor_test.cc: parameters, hashes, block write order
    st = src("pentago/data/supertensor_test.cc")
    sec = numbers(re.search(r"const section_t section\(\{(.*?)\}\);", st, re.S).group(1))
    order_blocks = numbers(re.search(r"ASSERT_EQ\(blocks, vec<uint16_t>\((.*?)\)\)", st).group(1))
    blocks = (ctypes.c_int * 4)(*order_blocks)
    order = np.zeros(4 * int(np.prod(order_blocks)), np.uint8)
    n = R.lib.ref_block_write_order(blocks, ctypes.c_void_p(order.ctypes.data))
    json.dump({"section": [sec[0:2], sec[2:4], sec[4:6], sec[6:8]],
               "block_size": numbers(re.search(r"const int block_size = (\d+);", st).group(1))[0],
               "filter": numbers(re.search(r"const int filter = (\d+);", st).group(1))[0],
               "level": numbers(re.search(r"const int level = (\d+);", st).group(1))[0],
               "key": numbers(re.search(r"uint128_t key = (\d+);", st).group(1))[0],
               "blocks": order_blocks,
               "write_order": order[:4 * n].reshape(-1, 4).tolist(),
               "sha1": re.findall(r'hash == "([0-9a-f]{40})"', st)},
              open(os.path.join(HERE, "supertensor.json"), "w"), indent=1)

    # 8. the solved database of slices 0..5 and its counts
    import shutil
    os.makedirs(os.path.join(HERE, "db"), exist_ok=True)
    for s in range(6):
        shutil.copyfile(os.path.join(ref_root, "data", f"slice-{s}.pentago"),
                        os.path.join(HERE, "db", f"slice-{s}.pentago"))
        shutil.copyfile(os.path.join(ref_root, "data", f"slice-{s}.pentago.index"),
                        os.path.join(HERE, "db", f"slice-{s}.pentago.index"))
    # sizes of the index files whose slices are not copied (slice 6) or not
    # shipped with the reference (slices 7 and 8)
    json.dump({str(s): os.path.getsize(os.path.join(ref_root, "data", f"slice-{s}.pentago.index"))
               for s in (6, 7, 8)}, open(os.path.join(HERE, "index_sizes.json"), "w"))
    # 9. shard samples and entry counts
    sh = src("pentago/shard/sharder_test.cc")
    pairs = re.findall(r"\{(\d+),(-?\d+)\}", re.search(r"server_values = \{(.*?)\};", sh, re.S).group(1))
    fixture = re.search(r"class shard_iterator_test.*?max_slice = (\d+);.*?total_shards = (\d+);", sh, re.S)
    shard_id = int(re.search(r"TEST_F\(shard_iterator_test, correctness\) \{\s*const int shard_id = (\d+);", sh).group(1))
    perm = src("pentago/shard/shard_permute.h")
    totals = [int(n) for n in re.findall(r"\{(\d+), \{[\d,]+\}\},\s*// slice", perm)]
    json.dump({"max_slice": int(fixture.group(1)), "total_shards": int(fixture.group(2)), "shard_id": shard_id,
               "server_values": [[int(b), int(v)] for b, v in pairs], "slice_totals": totals},
              open(os.path.join(HERE, "shards.json"), "w"))
    np.savez_compressed(os.path.join(HERE, "counts_0_5.npz"),
                        **{f"counts_{s}": np.load(os.path.join(ref_root, "data", f"counts-{s}.npy")) for s in range(6)})
    # 10. counts of the deep root's sections at slices 28 and 29
    deep_root_counts(ref_root)
    # 11. slice totals of end_test.cc
    et = src("pentago/end/end_test.cc")
    m = re.search(r"TEST\(end, simple_partition\) \{.*?stones = (\d+);\s*const uint64_t total = (\d+),\s*"
                  r"total_blocks = (\d+);.*?total_lines = (\d+);", et, re.S)
    json.dump({"slice": int(m.group(1)), "nodes": int(m.group(2)), "blocks": int(m.group(3)),
               "lines": int(m.group(4))}, open(os.path.join(HERE, "end_totals.json"), "w"))
    print("wrote fixtures to", HERE)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PENTAGO_REFERENCE", "/root/reference"))
