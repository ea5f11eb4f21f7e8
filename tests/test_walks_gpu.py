"""Random walks on the GPU (parw2v_random_walks), against a numpy restatement of the same
counter-based rule: walk w starts at node w mod n_nodes; step s moves to neighbour
(hi32(h) * degree) >> 32 of the current node, h = mix64(seed ^ mix64(w * 2^20 + s)).  Walks must be
identical, every step must follow an edge, a node without neighbours repeats, and the choice
among a node's neighbours is uniform."""
import numpy as np
import pytest

import par_word2vec_b200 as pw

pytestmark = pytest.mark.gpu

M64 = (1 << 64) - 1


def mix64(z):
    z = (z + 0x9E3779B97F4A7C15) & M64
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
    return z ^ (z >> 31)


def walks_restated(indptr, indices, walks_per_node, walk_len, seed):
    n = len(indptr) - 1
    out = np.empty((walks_per_node * n, walk_len), np.int32)
    for w in range(walks_per_node * n):
        v = w % n
        out[w, 0] = v
        for s in range(1, walk_len):
            lo, deg = int(indptr[v]), int(indptr[v + 1] - indptr[v])
            if deg > 0:
                h = mix64(seed ^ mix64(((w << 20) + s) & M64))
                v = int(indices[lo + (((h >> 32) * deg) >> 32)])
            out[w, s] = v
    return out


def random_graph(n, m, seed):
    rng = np.random.default_rng(seed)
    u, v = rng.integers(0, n, m), rng.integers(0, n, m)
    keep = u != v
    src = np.concatenate([u[keep], v[keep]])
    dst = np.concatenate([v[keep], u[keep]])
    order = np.argsort(src, kind="stable")
    indptr = np.zeros(n + 1, np.int64)
    np.add.at(indptr, src + 1, 1)
    return np.cumsum(indptr), dst[order].astype(np.int32)


def test_walks_match_restatement_and_follow_edges():
    indptr, indices = random_graph(200, 600, 1)
    # node 199 loses its edges: walks through it stop there
    cut = indices != 199
    src = np.repeat(np.arange(200), np.diff(indptr))[cut]
    indices = indices[cut]
    keep = src != 199
    src, indices = src[keep], indices[keep]
    indptr = np.zeros(201, np.int64)
    np.add.at(indptr, src + 1, 1)
    indptr = np.cumsum(indptr)
    got = pw.random_walks(indptr, indices, walks_per_node=3, walk_len=40, seed=12345)
    want = walks_restated(indptr, indices, 3, 40, 12345)
    assert np.array_equal(got, want)
    adj = set(zip(np.repeat(np.arange(200), np.diff(indptr)).tolist(), indices.tolist()))
    for w in got[:200]:
        for a, b in zip(w[:-1].tolist(), w[1:].tolist()):
            assert (a, b) in adj or (a == b and indptr[a + 1] == indptr[a])
    assert (got[199::200] == 199).all()  # the walks that start at the isolated node stay there


def test_neighbour_choice_is_uniform():
    # a star: node 0 joined to nodes 1..50; two-step walks from node 0 pick each leaf equally often
    leaves = np.arange(1, 51, dtype=np.int32)
    indptr = np.concatenate([[0, 50], 50 + np.arange(1, 51)]).astype(np.int64)
    indices = np.concatenate([leaves, np.zeros(50, np.int32)])
    got = pw.random_walks(indptr, indices, walks_per_node=4000, walk_len=2, seed=7)
    first = got[::51, 1]  # walks starting at node 0
    counts = np.bincount(first, minlength=51)[1:]
    expected = len(first) / 50
    chi2 = float(((counts - expected) ** 2 / expected).sum())
    assert chi2 < 90.0  # 49 degrees of freedom: p ~ 3e-4 beyond this


def test_walk_arguments_are_checked():
    with pytest.raises(pw.ParW2VError) as e:
        pw.random_walks(np.array([0, 1], np.int64), np.array([5], np.int32), 1, 4)
    assert e.value.status == pw.ERR_ARG
    with pytest.raises(pw.ParW2VError):
        pw.random_walks(np.array([0, 2, 1], np.int64), np.array([1, 0], np.int32), 1, 4)
