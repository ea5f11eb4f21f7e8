"""Hogwild modes against the reference CPU Hogwild run on the same corpus.

Bar (statistical, since Hogwild runs are not reproducible even on the reference; the reference is
run five times and its mean is the bar):
  final SGNS loss on a fixed evaluation set within 1% of the reference's, and planted-topic
  recall@10 within 0.01 of the reference's.
The reference is oracle/_ref/par_w2v_ref_fast (the reference source) at 16 threads, a fixed count: its own loss moves with the thread count."""
import os
import shutil
import subprocess
import tempfile

import numpy as np
import pytest

import par_word2vec_b200 as pw
from par_word2vec_b200 import evaluate, synth
from oracle import pwo

pytestmark = pytest.mark.gpu

REF_RUNS = 5
FLAGS = dict(size=100, window=5, negative=5, sample="1e-4", iter=1, min_count=5, batch_size=24, alpha="0.025")
N_TOPICS = 64


@pytest.fixture(scope="module")
def text_run():
    if not os.path.exists(pwo.REF_FAST_BIN):
        pytest.skip("reference not built (make -C oracle ref)")
    tmp = tempfile.mkdtemp()
    toks, lens = synth.topic_zipf(3000, 12000, N_TOPICS, doc_len=1000, seed=21)
    corpus = os.path.join(tmp, "c.txt")
    synth.write_text(corpus, toks, lens)
    threads = "16"  # the reference's Hogwild loss depends on its thread count: fixed, not the box's cores
    refs = []
    for run in range(REF_RUNS):  # the reference's Hogwild loss varies run to run: its mean is the bar
        args = [pwo.REF_FAST_BIN, "-train", corpus, "-output", os.path.join(tmp, "o.txt"), "-debug", "0",
                "-threads", threads, "-binary", "1", "-dump", os.path.join(tmp, "r")]
        for k, v in FLAGS.items():
            args += ["-" + k.replace("_", "-"), str(v)]
        subprocess.run(args, check=True, cwd=tmp, stdout=subprocess.DEVNULL)
        V, d, _, _ = map(int, open(os.path.join(tmp, "r.meta")).read().split())
        refs.append((np.fromfile(os.path.join(tmp, "r.win"), np.float32).reshape(V, d),
                     np.fromfile(os.path.join(tmp, "r.wout"), np.float32).reshape(V, d)))
    vocab = pw.Vocab.learn(corpus, FLAGS["min_count"])
    stream = vocab.load_stream(corpus)
    words = vocab.words()
    counts = vocab.counts()
    labels = evaluate.labels_from_words(words, N_TOPICS)
    queries = evaluate.top_queries(counts, labels, 3000)
    triples = evaluate.eval_triples(stream, counts, n_windows=4096)
    run = dict(tmp=tmp, V=V, d=d, stream=stream, counts=counts, labels=labels, queries=queries, triples=triples)
    scores = np.array([score(run, ri, ro) for ri, ro in refs])
    run.update(ref_loss=float(scores[:, 0].mean()), ref_recall=float(scores[:, 1].mean()),
               ref_losses=scores[:, 0].tolist())
    yield run
    shutil.rmtree(tmp)


def score(run, w_in, w_out):
    with pw.Trainer(size=run["d"], mode=pw.MODE_PLAIN) as t:
        t.set_vocab(run["counts"])
        t.set_weights(w_in, w_out)
        loss = evaluate.sgns_loss(t, run["triples"])
    rec = evaluate.recall_at_10(w_in, run["labels"], run["queries"], device="cuda")
    return loss, rec


def train_mode(run, mode, seed=1, variant=0):
    with pw.Trainer(mode=mode, seed=seed, variant=variant, size=FLAGS["size"], window=FLAGS["window"], negative=FLAGS["negative"],
                    batch_size=FLAGS["batch_size"], iter=FLAGS["iter"], alpha=float(FLAGS["alpha"]),
                    sample=float(FLAGS["sample"])) as t:
        t.set_vocab(run["counts"])
        t.init_weights()
        t.set_corpus(run["stream"])
        st = t.train()
        w_in, w_out = t.get_weights()
    return st, w_in, w_out


@pytest.mark.parametrize("mode,variant", [(pw.MODE_PLAIN, 0), (pw.MODE_BATCHED, pw.VARIANT_WINDOW),
                                          (pw.MODE_BATCHED, pw.VARIANT_STREAM),
                                          (pw.MODE_BATCHED_BF16, pw.VARIANT_WINDOW),
                                          (pw.MODE_BATCHED_BF16, pw.VARIANT_STREAM)])
def test_hogwild_matches_reference_loss_and_recall(text_run, mode, variant):
    ref_loss, ref_rec = text_run["ref_loss"], text_run["ref_recall"]
    st, w_in, w_out = train_mode(text_run, mode, variant=variant)
    assert np.isfinite(w_in).all() and np.isfinite(w_out).all()
    assert st["words"] == len(text_run["stream"])
    loss, rec = score(text_run, w_in, w_out)
    init_in, init_out = pwo.init_net(text_run["V"], text_run["d"])
    init_loss, _ = score(text_run, init_in, init_out)
    print(f"mode {mode} variant {variant}: loss {loss:.5f} (ref mean {ref_loss:.5f} of {text_run['ref_losses']}, init {init_loss:.5f}) recall {rec:.4f} (ref {ref_rec:.4f}) "
          f"kept {st['kept']} ms {st['kernel_ms']:.1f}")
    assert ref_loss < init_loss  # the evaluation set measures training
    assert abs(loss - ref_loss) <= 0.01 * ref_loss
    assert abs(rec - ref_rec) <= 0.01


def test_hogwild_stats_are_consistent(text_run):
    st, _, _ = train_mode(text_run, pw.MODE_PLAIN)
    n = len(text_run["stream"])
    assert st["words"] == n
    # subsampling keeps a fraction of the non-"</s>" tokens, each kept token is one position
    assert 0 < st["kept"] < n
    assert st["sentences"] > 0 and st["pairs"] > st["kept"]
    assert st["negatives"] % FLAGS["negative"] == 0
