"""The adaptive exact tier of a min-cut graph (the reference's EdgeStore, src/edge_store.cpp:60-300):
a graph that starts with few or no sketched levels keeps the deeper edges exactly and turns the store's
lowest level into a sketch level whenever the store reaches its budget.  Sketch levels end bit-identical
to levels sketched from the start (XOR linearity: a contracted level gets the present stored edges,
which equal all their toggles), the store holds exactly the present edges past the sketched levels, and
the min-cut driver answers from whatever is sketched at query time."""
import numpy as np
import pytest

import gpusketch_b200 as gs

pytestmark = pytest.mark.gpu


def _tags(restatement, edges, seed, L):
    return np.array([restatement.depth((int(a) << 32) | int(b), seed, L - 1) for a, b in edges.tolist()], np.int64)


def _expected_levels(restatement, V, seed, L, levels, initial, budget, calls):
    """Replays the contraction rule after every ingest call: while the present edges with tag >= first
    number at least `budget` and a level is free, first grows by one."""
    first, seen = initial, []
    for c in calls:
        seen.append(c)
        present = restatement.final_edges(V, np.concatenate(seen))
        tags = _tags(restatement, present, seed, L)
        while first < levels and int((tags >= first).sum()) >= budget:
            first += 1
    return first


@pytest.mark.parametrize("initial", [0, 1])
def test_adaptive_store_contracts_and_levels_stay_bit_exact(restatement, initial):
    V, seed, levels, L = 700, 0x5EED5000, 4, 19
    rng = np.random.default_rng(50 + initial)
    base = rng.integers(0, V, size=(24000, 2), dtype=np.uint32)
    pairs = np.concatenate([base, base[:3000], rng.integers(0, V, size=(12000, 2), dtype=np.uint32)])
    calls = np.array_split(pairs, 7)
    budget = 2500
    with gs.GraphSketch(V, seed, num_levels=levels, num_subgraphs=L) as g:
        g.set_edge_store(initial, 16 * budget)
        assert g.sketched_levels() == (initial, 0)
        for c in calls:
            g.ingest_pairs(c)
        first, contractions = g.sketched_levels()
        assert first == _expected_levels(restatement, V, seed, L, levels, initial, budget, calls)
        assert contractions == first - initial and first > initial
        sk = restatement.new_sketches(V, levels=levels)
        restatement.ingest_levels(sk, V, levels, L, seed, pairs)
        nb = restatement.geometry(V)["num_buckets"]
        for lv in range(levels):
            got = g.download(lv).tobytes()
            if lv < first:
                assert got == sk[lv * V * nb * 2:(lv + 1) * V * nb * 2].tobytes(), lv
            else:
                assert not np.frombuffer(got, np.uint64).any(), lv
        final = restatement.final_edges(V, pairs)
        want = final[_tags(restatement, final, seed, L) >= first]
        want = want[np.lexsort((want[:, 1], want[:, 0]))]
        assert np.array_equal(g.edge_store_edges(), want)
        # clearing returns to the initial levels
        g.clear()
        assert g.sketched_levels()[0] == initial and len(g.edge_store_edges()) == 0
        with pytest.raises(gs.GpuSketchError):
            g.ingest_pairs(calls[0])
            g.set_edge_store(initial, 0)                      # only before the first ingest


def _planted(n, seed, p=0.3, cut=3):
    rng = np.random.default_rng(seed)
    blocks = []
    for off in (0, n):
        a, b = np.triu_indices(n, 1)
        keep = rng.random(a.size) < p
        blocks.append(np.stack([a[keep] + off, b[keep] + off], 1))
    cross = np.stack([rng.integers(0, n, cut), rng.integers(n, 2 * n, cut)], 1)
    pairs = np.concatenate(blocks + [cross]).astype(np.uint32)
    return pairs[rng.permutation(len(pairs))]


@pytest.mark.parametrize("initial,budget", [(0, 10**9), (0, 2000), (1, 1500)])
def test_min_cut_over_the_adaptive_store(initial, budget):
    """All exact (no contraction: the exact tier answers at level 0), and contracted into sketch
    levels before the query (a sketched level certifies the planted cut): the min cut is 3 either way."""
    n, seed = 150, 0x5EED5001
    pairs = _planted(n, 13)
    V = 2 * n
    L = 1 + 2 * int(np.log2(V))
    with gs.GraphSketch(V, seed, num_levels=4, num_subgraphs=L) as g:
        g.set_edge_store(initial, 16 * budget)
        for c in np.array_split(pairs, 5):
            g.ingest_pairs(c)
        first, _ = g.sketched_levels()
        value, level, cut_at, side = g.min_cut(4)
        assert value == 3
        if first == 0:
            assert level == 0 and cut_at == 3      # answered by the exact tier
        else:
            assert level < first
        s = side.astype(bool)
        assert (s[:n].all() or not s[:n].any()) and (s[n:].all() or not s[n:].any()) and s[0] != s[n]
