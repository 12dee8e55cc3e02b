"""The tree oracle (oracle/tree_oracle.c) against a second, independently written restatement.

No reference test pins the diff's byte order, the shifted-duplicate sources or the region
choices (its atomics permute them); they follow from the reference source executed one thread
at a time.  This file restates that execution a second time, as plain Python loops over small
trees, directly from the reference functions:

* dedup_data_baseline  src/tree_approach.cpp:13-259 (leaf labels against a fresh all-zero tree,
  lowest-index first occurrence, first-occurrence forest, region selection level by level with
  the level's digests inserted after its region pass);
* dedup_data           src/tree_approach.cpp:261-509 (the same with the prior tree and map;
  shifted-duplicate parents hashed before their existence test);
* collect_diff         src/tree_approach.cpp:511-710 (first regions in push order, repeat table
  ascending by source checkpoint, shift rows stably grouped by source checkpoint, region data
  zero-padded to whole chunks);
* checkpoint           src/tree_approach.cpp:1577-1689 (a baseline starts from a new tree and
  map; checkpoint ids keep counting).

Chunk and node digests come from the oracle's hash (pinned separately by the reference's hash
vectors); everything else here is independent of the C oracle.
"""
import struct

import numpy as np
import pytest

from oracle import oracle as O

FIRST, FIXED, SHIFT, DONE = 0, 1, 2, 4
ZERO = bytes(16)


def deepest_range(node, num_nodes):
    """(leftmost, rightmost) heap indices under `node` on the deepest level that exists
    (include/kokkos_merkle_tree.hpp:102-129), including the clamp that drops a shallower
    straddled level"""
    lo, hi = 2 * node + 1, 2 * node + 2
    while lo < num_nodes:
        lo, hi = 2 * lo + 1, 2 * hi + 2
    lo, hi = (lo - 1) // 2, (hi - 2) // 2
    if hi > num_nodes:
        hi = num_nodes - 1
    return lo, hi


def level_ranges(num_nodes):
    """heap levels from below the deepest one up to the root, as the reference's
    level_beg/level_end loop walks them"""
    ranges = []
    beg = end = 0
    while end < num_nodes:
        beg, end = 2 * beg + 1, 2 * end + 2
    while True:
        ranges.append((beg, end))
        if beg == 0:
            return ranges
        beg, end = (beg - 1) // 2, (end - 2) // 2


class PyTreeModel:
    def __init__(self, cs, kind):
        self.cs, self.kind = cs, kind
        self.current_id = 0
        self.baseline_id = 0
        self.tree = []
        self.map = {}          # digest -> [node, checkpoint]

    def h(self, b):
        return O.hash_bytes(bytes(b), self.kind)

    def insert(self, d, node):
        if d in self.map:
            return False
        self.map[d] = [node, self.current_id]
        return True

    def checkpoint(self, data, make_baseline):
        data = bytes(data)
        n = -(-len(data) // self.cs)
        N = 2 * n - 1
        baseline = make_baseline or self.current_id == 0
        if baseline:
            self.tree = [ZERO] * N
            self.map = {}
            self.baseline_id = self.current_id
        cur = self.current_id
        tree, lab = self.tree, [DONE] * N
        first, shift = [], []

        # leaves, one after another in ascending order
        for leaf in range(n - 1, N):
            off = (leaf - (n - 1)) * self.cs
            d = self.h(data[off:off + self.cs])
            new = self.insert(d, leaf)
            if d == tree[leaf]:
                lab[leaf] = FIXED
            elif new:
                lab[leaf] = FIRST
            else:
                e = self.map[d]
                if e[1] == cur:
                    e[0] = min(e[0], leaf)
                    lab[leaf] = FIRST
                else:
                    lab[leaf] = SHIFT
            if baseline or lab[leaf] != FIXED:
                tree[leaf] = d
        for leaf in range(n - 1, N):
            if lab[leaf] == FIRST:
                e = self.map[tree[leaf]]
                if e[1] == cur and e[0] != leaf:
                    lab[leaf] = SHIFT

        inner = lambda beg, end: [v for v in range(beg, end + 1) if v < n - 1]
        # first-occurrence forest
        for beg, end in level_ranges(N):
            for v in inner(beg, end):
                l, r = 2 * v + 1, 2 * v + 2
                if lab[l] == FIRST and lab[r] == FIRST:
                    lab[v] = FIRST
                    tree[v] = self.h(tree[l] + tree[r])
                    self.insert(tree[v], v)
                if v == 0 and lab[0] == FIRST:
                    first.append(0)
        # region selection
        for beg, end in level_ranges(N):
            for v in inner(beg, end):
                l, r = 2 * v + 1, 2 * v + 2
                if lab[l] != lab[r]:
                    lab[v] = DONE
                    for c in (l, r):
                        if lab[c] == SHIFT:
                            shift.append(c)
                        elif lab[c] != FIXED and lab[c] != DONE:
                            first.append(c)
                elif lab[l] == FIXED:
                    lab[v] = FIXED
                elif lab[l] == SHIFT:
                    if not baseline:
                        tree[v] = self.h(tree[l] + tree[r])
                    if tree[v] in self.map:
                        lab[v] = SHIFT
                    else:
                        lab[v] = DONE
                        shift += [l, r]
            if baseline:
                for v in inner(beg, end):
                    tree[v] = self.h(tree[2 * v + 1] + tree[2 * v + 2])
                    self.insert(tree[v], v)

        diff = self.collect(data, n, N, first, shift)
        self.current_id += 1
        return diff

    def collect(self, data, n, N, first, shift):
        cur, tree = self.current_id, self.tree
        regions = []
        for v in first:
            e = self.map[tree[v]]
            if e == [v, cur]:
                regions.append(v)
        leaves = []
        for v in regions:
            lo, hi = deepest_range(v, N)
            leaves += [lo - (n - 1) + j for j in range(hi - lo + 1)]
        src = [self.map[tree[v]] for v in shift]
        counts = [0] * (cur + 1)
        for _, t in src:
            counts[t] += 1
        rows = [(t, c) for t, c in enumerate(counts) if c]
        order = sorted(range(len(shift)), key=lambda i: src[i][1])      # stable
        meta = bytearray(4 * len(first))
        for i, v in enumerate(regions):
            meta[4 * i:4 * i + 4] = struct.pack("<I", v)
        meta += b"".join(struct.pack("<II", t, c) for t, c in rows)
        meta += b"".join(struct.pack("<II", shift[i], src[i][0]) for i in order)
        body = b"".join(data[c * self.cs:(c + 1) * self.cs].ljust(self.cs, b"\0") for c in leaves)
        hdr = struct.pack("<IIQIIII", self.baseline_id, cur, len(data), self.cs, len(first), len(rows), len(shift))
        return hdr + bytes(meta) + body


def series(rng, cs, n, size, steps):
    """buffers built from a small palette of chunk contents (many repeats), with whole runs
    reverted to earlier checkpoints and blocks copied to chunk-aligned offsets"""
    palette = rng.integers(0, 256, (5, cs), dtype=np.uint8)

    def fresh():
        pick = rng.integers(0, len(palette) + 3, n)
        return np.concatenate([palette[p] if p < len(palette) else rng.integers(0, 256, cs, dtype=np.uint8)
                               for p in pick])[:size]
    bufs = [fresh()]
    for _ in range(steps - 1):
        b = bufs[-1].copy()
        kind = rng.integers(0, 4)
        if kind == 0:
            b = fresh()
        elif kind == 1 and len(bufs) > 1:
            k = int(rng.integers(0, len(bufs)))
            a, z = sorted(rng.integers(0, n + 1, 2))
            b[a * cs:z * cs] = bufs[k][a * cs:z * cs]
        else:
            for _ in range(int(rng.integers(1, 4))):
                a, z = sorted(rng.integers(0, n, 2))
                dst = int(rng.integers(0, n - (z - a) + 1))
                blk = b[a * cs:(z + 1) * cs].copy()
                b[dst * cs:dst * cs + len(blk)] = blk[:len(b) - dst * cs]
                c = int(rng.integers(0, n))
                b[c * cs:(c + 1) * cs] = rng.integers(0, 256, len(b[c * cs:(c + 1) * cs]), dtype=np.uint8)
        bufs.append(b)
    return bufs


@pytest.mark.parametrize("seed,steps,rebase", [(s, 7, True) for s in range(10)] + [(10, 14, False), (11, 14, False)])
def test_tree_oracle_matches_independent_model(seed, steps, rebase):
    """single-chunk to 257-chunk trees, full and ragged last chunks, both hashes; series with
    baselines mid-sequence, and two 14-checkpoint chains whose shift rows reach back over many
    checkpoints"""
    rng = np.random.default_rng(100 + seed)
    cs = [16, 32, 64, 48, 16, 128, 32, 64, 16, 24, 32, 16][seed]
    kind = O.HASH_MD5 if seed % 3 == 2 else O.HASH_MURMUR3
    n = [1, 2, 3, 8, 64, 100, 5, 128, 257, 33, 96, 200][seed]
    size = n * cs - (int(rng.integers(0, cs)) if seed % 2 else 0)
    bufs = series(rng, cs, n, size, steps)
    baselines = [True] + [rebase and bool(rng.integers(0, 5) == 0) for _ in range(steps - 1)]
    o = O.OracleTreeDeduplicator(cs, kind)
    m = PyTreeModel(cs, kind)
    for i, (b, mb) in enumerate(zip(bufs, baselines)):
        want = m.checkpoint(b, mb)
        got = o.checkpoint(b, mb)
        assert got == want, (seed, i)
    o.close()


def test_model_matches_reference_test_case_counts():
    """the model itself against the reference's own expectations (test/test_case_*.cpp: the
    first-occurrence and shifted-duplicate region counts of the second checkpoint), and against
    the committed diffs of those cases"""
    import json
    import os

    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "test_cases.json")) as f:
        cases = json.load(f)
    for name, c in cases.items():
        m = PyTreeModel(1, O.HASH_MURMUR3)
        d0 = m.checkpoint(c["step0"].encode(), True)
        d1 = m.checkpoint(c["step1"].encode(), False)
        F, S = struct.unpack("<II", d1[20:24] + d1[28:32])
        assert (F, S) == (c["first"], c["shift"]), name
        assert d0.hex() == c["diff0"] and d1.hex() == c["diff1"], name
