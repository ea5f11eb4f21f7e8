"""The text8-shaped workload: 17,000 documents of 1,000 tokens (17M tokens) over 71,290 types,
64 planted topics, each token from a global Zipf(1.0) with p = 0.5 and from its document topic's
Zipf(1.0) slice otherwise; d = 100, window 5, 5 negatives, sample 1e-4, min-count 5, 1 iteration.

Hogwild modes against the reference CPU Hogwild run (the mean of five runs at 16 threads):
final SGNS loss on a fixed evaluation set within 1%, planted-topic recall@10 within 0.01."""
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
N_TOPICS = 64
FLAGS = dict(size=100, window=5, negative=5, sample="1e-4", iter=1, min_count=5, batch_size=24, alpha="0.025")


def score(run, w_in, w_out):
    with pw.Trainer(size=run["d"], mode=pw.MODE_PLAIN) as t:
        t.set_vocab(run["counts"])
        t.set_weights(w_in, w_out)
        loss = evaluate.sgns_loss(t, run["triples"])
    return loss, evaluate.recall_at_10(w_in, run["labels"], run["queries"], device="cuda")


@pytest.fixture(scope="module")
def text8_run():
    if not os.path.exists(pwo.REF_FAST_BIN):
        pytest.skip("reference not built (make -C oracle ref)")
    tmp = tempfile.mkdtemp()
    toks, lens = synth.topic_zipf(17000, 71290, N_TOPICS, doc_len=1000, seed=1)
    corpus = os.path.join(tmp, "text8_like.txt")
    synth.write_text(corpus, toks, lens)
    refs = []
    for _ in range(REF_RUNS):  # the reference's Hogwild loss varies run to run: its mean is the bar
        args = [pwo.REF_FAST_BIN, "-train", corpus, "-output", os.path.join(tmp, "o.txt"), "-debug", "0",
                "-threads", "16", "-binary", "1", "-dump", os.path.join(tmp, "r")]
        for k, v in FLAGS.items():
            args += ["-" + k.replace("_", "-"), str(v)]
        subprocess.run(args, check=True, cwd=tmp, stdout=subprocess.DEVNULL)
        V, d, _, _ = map(int, open(os.path.join(tmp, "r.meta")).read().split())
        refs.append((np.fromfile(os.path.join(tmp, "r.win"), np.float32).reshape(V, d),
                     np.fromfile(os.path.join(tmp, "r.wout"), np.float32).reshape(V, d)))
    vocab = pw.Vocab.learn(corpus, FLAGS["min_count"])
    stream = vocab.load_stream(corpus)
    counts = vocab.counts()
    labels = evaluate.labels_from_words(vocab.words(), N_TOPICS)
    run = dict(d=d, stream=stream, counts=counts, labels=labels,
               queries=evaluate.top_queries(counts, labels, 10000),
               triples=evaluate.eval_triples(stream, counts, n_windows=4096))
    scores = np.array([score(run, ri, ro) for ri, ro in refs])
    run.update(ref_loss=float(scores[:, 0].mean()), ref_recall=float(scores[:, 1].mean()),
               ref_losses=scores[:, 0].tolist())
    yield run
    shutil.rmtree(tmp)


@pytest.mark.parametrize("mode", [pw.MODE_PLAIN, pw.MODE_BATCHED_BF16])
def test_text8_matches_reference_loss_and_recall(text8_run, mode):
    run = text8_run
    with pw.Trainer(mode=mode, seed=1, size=FLAGS["size"], window=FLAGS["window"], negative=FLAGS["negative"],
                    batch_size=FLAGS["batch_size"], iter=FLAGS["iter"], alpha=float(FLAGS["alpha"]),
                    sample=float(FLAGS["sample"])) as t:
        t.set_vocab(run["counts"])
        t.init_weights()
        t.set_corpus(run["stream"])
        st = t.train()
        w_in, w_out = t.get_weights()
    assert np.isfinite(w_in).all() and np.isfinite(w_out).all()
    assert st["words"] == len(run["stream"])
    loss, rec = score(run, w_in, w_out)
    print(f"text8 mode {mode}: loss {loss:.5f} (ref mean {run['ref_loss']:.5f} of {run['ref_losses']}) "
          f"recall {rec:.4f} (ref {run['ref_recall']:.4f}) ms {st['kernel_ms']:.1f}")
    assert abs(loss - run["ref_loss"]) <= 0.01 * run["ref_loss"]
    assert abs(rec - run["ref_recall"]) <= 0.01
