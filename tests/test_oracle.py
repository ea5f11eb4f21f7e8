"""The C restatement (oracle/) is pinned to the reference's own outputs (tests/golden)."""
import hashlib

import numpy as np

from oracle import pwo


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def test_exp_table_matches_reference(golden):
    assert np.array_equal(bits(pwo.exp_table()), bits(golden.exptable))


def test_unigram_table_matches_reference(golden):
    t = pwo.unigram_table(golden.counts)
    assert hashlib.sha256(t.tobytes()).hexdigest() == golden.meta["table_sha256"]


def test_init_net_matches_reference(golden):
    w_in, w_out = pwo.init_net(len(golden.counts), int(golden.flags["size"]))
    assert hashlib.sha256(w_in.tobytes()).hexdigest() == golden.meta["win0_sha256"]
    assert not w_out.any()


def test_stream_length_is_train_words(golden):
    # loadStream at one thread reads every in-vocabulary token: train_words of them + sentinel
    assert len(golden.stream) - 1 == golden.meta["train_words"] == int(golden.counts.sum())
    assert golden.stream[-1] == 0


def test_training_loop_bit_exact(golden):
    V, d = len(golden.counts), int(golden.flags["size"])
    w_in, w_out = pwo.init_net(V, d)
    tr = pwo.train(golden.counts, golden.stream, w_in, w_out, **golden.train_kwargs())
    assert tr["rc"] == 0
    assert np.array_equal(bits(w_in), bits(golden.win))
    assert np.array_equal(bits(w_out), bits(golden.wout))


def test_trace_is_consistent(golden):
    V, d = len(golden.counts), int(golden.flags["size"])
    w_in, w_out = pwo.init_net(V, d)
    caps = dict(keep=10**6, b=10**6, alpha=10**6, rep_b=10**6, neg=10**6)
    tr = pwo.train(golden.counts, golden.stream, w_in, w_out, trace_caps=caps, **golden.train_kwargs())
    k = golden.train_kwargs()
    # every token is read once per epoch, plus the sentinel that ends each epoch
    assert tr["n_keep"] == k["iter"] * len(golden.stream)
    assert tr["words_read"] == k["iter"] * len(golden.stream)
    assert (tr["b"] < k["window"]).all() and (tr["rep_b"] < 2 * k["window"]).all()
    assert tr["n_neg"] == int(tr["rep_b"].astype(np.int64).sum()) * k["negative"]
    assert ((tr["neg"] > 0) & (tr["neg"] < V)).all()
    assert (tr["alpha"] <= k["alpha"]).all() and (tr["alpha"] >= k["alpha"] * 1e-4 * 0.999).all()


def test_planted_mistake_is_caught(golden):
    """A one-ulp change of the oracle's inputs must break bit-equality (the check has teeth)."""
    V, d = len(golden.counts), int(golden.flags["size"])
    w_in, w_out = pwo.init_net(V, d)
    w_in[1, 0] = np.nextafter(w_in[1, 0], np.float32(1))
    pwo.train(golden.counts, golden.stream, w_in, w_out, **golden.train_kwargs())
    assert not np.array_equal(bits(w_in), bits(golden.win))


def test_window_variant_is_deterministic_and_trains(golden_cases):
    g = golden_cases["d100"]
    V, d = len(g.counts), int(g.flags["size"])
    runs = []
    for _ in range(2):
        w_in, w_out = pwo.init_net(V, d)
        tr = pwo.train(g.counts, g.stream, w_in, w_out, sync_window=1, **g.train_kwargs())
        assert tr["rc"] == 0
        runs.append((w_in, w_out))
    assert np.array_equal(bits(runs[0][0]), bits(runs[1][0]))
    assert np.isfinite(runs[0][0]).all()
    rel = np.linalg.norm(runs[0][0] - g.win) / np.linalg.norm(g.win)
    assert 0 < rel < 0.5  # a different trajectory, same scale as the reference's
