"""DET mode on the GPU against the reference (tests/golden) and the oracle's trace.

Bar: bit-exact.  The unigram table, expTable and InitNet are byte-equal; after training,
W_in and W_out have the reference's bit patterns; every random decision (keep/drop, b, rep_b,
negative ids) equals the oracle's trace."""
import hashlib

import numpy as np
import pytest

import par_word2vec_b200 as pw
from oracle import pwo

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def make(golden, mode=pw.MODE_DET, **over):
    k = golden.train_kwargs()
    k.update(over)
    t = pw.Trainer(mode=mode, seed=0, **k)
    t.set_vocab(golden.counts)
    return t


def test_tables_on_device(golden):
    with make(golden) as t:
        assert hashlib.sha256(t.get_table().tobytes()).hexdigest() == golden.meta["table_sha256"]
        assert np.array_equal(bits(t.get_exp_table()), bits(golden.exptable))
        t.init_weights()
        w_in, w_out = t.get_weights()
        assert hashlib.sha256(w_in.tobytes()).hexdigest() == golden.meta["win0_sha256"]
        assert not w_out.any()


def test_det_training_bit_exact(golden):
    with make(golden) as t:
        t.init_weights()
        t.set_corpus(golden.stream[:-1])
        st = t.train()
        w_in, w_out = t.get_weights()
    k = golden.train_kwargs()
    assert st["words"] == k["iter"] * len(golden.stream)
    bad_in = int((bits(w_in) != bits(golden.win)).sum())
    bad_out = int((bits(w_out) != bits(golden.wout)).sum())
    assert bad_in == 0 and bad_out == 0, (bad_in, bad_out, float(np.abs(w_in - golden.win).max()))


def test_det_trace_equals_oracle(golden):
    caps = dict(keep=10**6, b=10**6, alpha=10**6, rep_b=10**6, neg=10**6)
    V, d = len(golden.counts), int(golden.flags["size"])
    w_in, w_out = pwo.init_net(V, d)
    ref = pwo.train(golden.counts, golden.stream, w_in, w_out, trace_caps=caps, **golden.train_kwargs())
    with make(golden) as t:
        t.init_weights()
        t.set_corpus(golden.stream[:-1])
        t.set_trace(keep_cap=caps["keep"], b_cap=caps["b"], alpha_cap=caps["alpha"], rep_b_cap=caps["rep_b"],
                    neg_cap=caps["neg"])
        t.train()
        tr = t.trace()
    for k in ("keep", "b", "rep_b", "neg"):
        assert tr["n_" + k] == ref["n_" + k], k
        assert np.array_equal(tr[k], ref[k]), k
    assert np.array_equal(bits(tr["alpha"]), bits(ref["alpha"]))
    assert tr["final_lcg"] == ref["final_lcg"]


def test_det_resume_from_weights_matches_fresh_run(golden_cases):
    """set_weights(init) + train == init_weights + train (the upload path is exact)."""
    g = golden_cases["text_small"]
    V, d = len(g.counts), int(g.flags["size"])
    w_in, w_out = pwo.init_net(V, d)
    with make(g) as t:
        t.set_weights(w_in, w_out)
        t.set_corpus(g.stream[:-1])
        t.train()
        a, b = t.get_weights()
    assert np.array_equal(bits(a), bits(g.win)) and np.array_equal(bits(b), bits(g.wout))


def test_resample_limit_reports_timeout():
    """Every vocabulary word occurs in the sentence: the reference would spin forever in its
    negative redraw loop (PAR_Word2Vec_cpu.cpp:611-615); the library gives up and says so."""
    counts = np.array([1, 50, 50, 50], np.uint32)
    stream = np.array([1, 2, 3] * 10 + [0], np.int32)
    with pw.Trainer(size=8, window=2, negative=3, batch_size=4, iter=1, alpha=0.025, sample=0,
                    mode=pw.MODE_DET) as t:
        t.set_vocab(counts)
        t.init_weights()
        t.set_corpus(stream)
        with pytest.raises(pw.ParW2VError) as e:
            t.train()
        assert e.value.status == pw.ERR_TIMEOUT
        # the context stays usable after the error
        t.set_corpus(np.array([1, 2, 0], np.int32))
        assert len(t.get_exp_table()) == 1001


def test_out_of_vocabulary_ids_rejected():
    with pw.Trainer(size=8, window=2, negative=2, batch_size=4, iter=1, mode=pw.MODE_DET) as t:
        t.set_vocab(np.array([3, 5, 5], np.uint32))
        t.init_weights()
        t.set_corpus(np.array([1, 2, 7, 0], np.int32))
        with pytest.raises(pw.ParW2VError) as e:
            t.train()
        assert e.value.status == pw.ERR_ARG


def test_call_order_errors():
    with pw.Trainer(size=8, mode=pw.MODE_DET) as t:
        with pytest.raises(pw.ParW2VError) as e:
            t.train()
        assert e.value.status == pw.ERR_STATE


def test_memory_cap_is_enforced():
    with pw.Trainer(size=8, mode=pw.MODE_PLAIN, mem_cap_bytes=64 << 20) as t:
        with pytest.raises(pw.ParW2VError) as e:
            t.set_vocab(np.array([3, 5, 5], np.uint32))  # the 400 MB table does not fit in 64 MB
        assert e.value.status == pw.ERR_OOM


def test_det_window_variant_bit_exact_vs_oracle(golden):
    """The window-synchronous attraction (the BATCHED modes' default) is pinned the same way:
    DET with PARW2V_ATTRACT_WINDOW equals the oracle's restatement of that variant bit for bit."""
    V, d = len(golden.counts), int(golden.flags["size"])
    w_in, w_out = pwo.init_net(V, d)
    pwo.train(golden.counts, golden.stream, w_in, w_out, sync_window=1, **golden.train_kwargs())
    with make(golden, attraction=pw.ATTRACT_WINDOW) as t:
        t.init_weights()
        t.set_corpus(golden.stream[:-1])
        t.train()
        a, b = t.get_weights()
    assert np.array_equal(bits(a), bits(w_in)) and np.array_equal(bits(b), bits(w_out))
    # and it is a different trajectory from the reference's sequential attraction
    assert not np.array_equal(bits(a), bits(golden.win))
