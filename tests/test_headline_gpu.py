"""Parity of the benchmark's workload -- the 1B-word-shaped corpus, batched BF16 and batched FP32 --
against the reference CPU Hogwild run.

Corpus: the generator the benchmark uses (topic-mixture Zipf(1.0) over 555,000 types with 256
planted topics, lognormal sentence lengths with mean 25 and sigma 1, seed 4; words under min-count
5 dropped).  d = 300, window 5, 5 negatives, sample 1e-4, batch 24, alpha 0.025, 1 iteration.

Two sizes, because at a fixed number of sentences in flight the loss moves with the corpus size
(concurrency acts like extra step size on frequent rows):
  * 100M tokens at the library's default cap on sentences in flight (lines / 8192, about 490);
    the reference is run three times at 16 threads and its mean is the bar;
  * the benchmark's own 800M-token corpus at the benchmark's concurrency (148 CTAs x 16 warps =
    2,368 sentences in flight: the default leaves this corpus uncapped); the reference takes about
    four minutes a run here, so it runs once.

The bar (PAR_Word2Vec_cpu.cpp:529-680 is the algorithm):
  * final SGNS loss on a fixed evaluation set within 1% of the reference's;
  * planted-topic recall@10 over the 10,000 most frequent words within 0.01 (saturated near 1);
  * the planted-topic margin (cosine to the own topic's centroid minus the mean cosine to the
    other centroids), a continuous measure where recall@10 saturates, within 10% of the
    reference's, for the 10,000 most frequent words and for the words of frequency rank 200,000 to
    400,000.
"""
import os
import shutil
import tempfile

import numpy as np
import pytest

import par_word2vec_b200 as pw
from par_word2vec_b200 import evaluate, synth
from oracle import pwo, ref_run

pytestmark = pytest.mark.gpu

N_TYPES, N_TOPICS = 555_000, 256
HYPER = dict(size=300, window=5, negative=5, batch_size=24, iter=1, alpha=0.025, sample=1e-4)
FLAGS = dict(size=300, window=5, negative=5, sample="1e-4", iter=1, min_count=5, batch_size=24, alpha="0.025")
REF_THREADS = 16


def rank_queries(counts: np.ndarray, labels: np.ndarray, lo: int, hi: int) -> np.ndarray:
    """Labelled words of frequency rank lo..hi (vocabulary rows are sorted by count)."""
    return evaluate.top_queries(counts, labels, hi)[lo:]


def score(run, w_in, w_out):
    with pw.Trainer(size=HYPER["size"], mode=pw.MODE_PLAIN) as t:
        t.set_vocab(run["counts"])
        t.set_weights(w_in, w_out)
        loss = evaluate.sgns_loss(t, run["triples"])
    top = evaluate.recall_at_10(w_in, run["labels"], run["queries"], device="cuda")
    m_top = evaluate.topic_margin(w_in, run["labels"], run["queries"], device="cuda")
    m_rare = evaluate.topic_margin(w_in, run["labels"], run["rare"], device="cuda")
    return loss, top, m_top, m_rare


def make_run(n_tokens: int, ref_runs: int):
    if not os.path.exists(pwo.REF_FAST_BIN):
        pytest.skip("reference not built (make -C oracle ref)")
    stream_d, counts, words, gen_ids = synth.topic_zipf_stream_torch(n_tokens, N_TYPES, N_TOPICS, seed=4,
                                                                     min_count=5, device="cuda")
    stream = stream_d.cpu().numpy()
    del stream_d
    labels = np.full(len(counts), -1, np.int64)
    labels[1:] = gen_ids % N_TOPICS
    tmp = tempfile.mkdtemp()
    corpus, vocab_file = os.path.join(tmp, "c.txt"), os.path.join(tmp, "c.vocab")
    synth.write_stream_text(corpus, stream, words)
    ref_run.write_vocab(vocab_file, words, counts)
    run = dict(stream=stream, counts=counts, labels=labels, tmp=tmp,
               queries=evaluate.top_queries(counts, labels, 10_000),
               rare=rank_queries(counts, labels, 200_000, min(400_000, len(counts) - 1)),
               triples=evaluate.eval_triples(stream, counts, n_windows=4096))
    scores = []
    for _ in range(ref_runs):
        r = ref_run.run(corpus, FLAGS, REF_THREADS, read_vocab=vocab_file)
        assert r["V"] == len(counts) and r["train_words"] == int(counts.sum())
        scores.append(score(run, *ref_run.rows_in_order(r, words)))
    os.remove(corpus)
    scores = np.array(scores)
    run.update(ref=scores.mean(axis=0), ref_all=scores.tolist())
    return run


@pytest.fixture(scope="module")
def run_100m():
    run = make_run(100_000_000, 3)
    yield run
    shutil.rmtree(run["tmp"])


@pytest.fixture(scope="module")
def run_800m():
    run = make_run(800_000_000, 1)
    yield run
    shutil.rmtree(run["tmp"])


def check(run, label, mode, **kw):
    with pw.Trainer(mode=mode, seed=1, **HYPER, **kw) as t:
        t.set_vocab(run["counts"])
        t.init_weights()
        t.set_corpus(run["stream"])
        st = t.train()
        w_in, w_out = t.get_weights()
    assert np.isfinite(w_in).all() and np.isfinite(w_out).all()
    assert st["words"] == len(run["stream"])
    loss, top, m_top, m_rare = score(run, w_in, w_out)
    ref_loss, ref_top, ref_m_top, ref_m_rare = run["ref"]
    print(f"{label} mode {mode} {kw} (grid {st['grid']} x {st['warps_per_cta']} warps, {st['lane_elems']} elements "
          f"per lane, staging {st['staging']}, attraction {st['attraction']}): loss {loss:.5f} (ref {ref_loss:.5f}, "
          f"{100 * (loss / ref_loss - 1):+.2f}%) recall@10 {top:.4f} (ref {ref_top:.4f}) topic margin {m_top:.4f} "
          f"(ref {ref_m_top:.4f}), rank 200k-400k {m_rare:.4f} (ref {ref_m_rare:.4f}); reference runs "
          f"{run['ref_all']}; kernel {st['kernel_ms']:.1f} ms, {st['words'] / st['kernel_ms'] / 1e3:.1f}M words/s")
    assert abs(loss - ref_loss) <= 0.01 * ref_loss
    assert abs(top - ref_top) <= 0.01
    assert abs(m_top - ref_m_top) <= 0.1 * abs(ref_m_top)
    assert abs(m_rare - ref_m_rare) <= 0.1 * abs(ref_m_rare)


@pytest.mark.parametrize("mode,autotune", [(pw.MODE_BATCHED_BF16, 0), (pw.MODE_BATCHED, 0), (pw.MODE_BATCHED_BF16, 1)])
def test_100m_default_concurrency_matches_reference(run_100m, mode, autotune):
    """autotune = 1: the launch knobs the autotuner picks leave the result within the same bars."""
    check(run_100m, "100M default", mode, autotune=autotune)


@pytest.mark.parametrize("mode", [pw.MODE_BATCHED_BF16, pw.MODE_BATCHED])
def test_bench_corpus_matches_reference(run_800m, mode):
    """The benchmark's corpus and concurrency (the default cap leaves 32M lines uncapped)."""
    check(run_800m, "800M bench", mode)
