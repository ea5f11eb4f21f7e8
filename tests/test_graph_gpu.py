"""Graph embedding (the PAR_Word2Vec_gpu_graph workload): Hogwild modes against the reference CPU
Hogwild run on uniform random walks over a degree-corrected stochastic block model.

Workload: 10,312 nodes in 39 communities, ~334k undirected edges (70% inside a community,
power-law degree propensities with exponent 2.5), 10 walks of length 80 from every node (8.25M
tokens); d = 128, window 10, 5 negatives, no subsampling, 1 iteration, batch 24.  Window 10 puts
up to 95 shared negatives in a batch, beyond the tensor-core tile, so the BF16 modes run the
CUDA-core repulsion here.

Bar, as for text: final SGNS loss on a fixed evaluation set within 1% of the reference's (the mean
of five runs of the reference at 16 threads), and
planted-community recall@10 (all nodes are queries) within 0.01 of the reference's."""
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
FLAGS = dict(size=128, window=10, negative=5, sample="0", iter=1, min_count=5, batch_size=24, alpha="0.025")


@pytest.fixture(scope="module")
def graph_run():
    if not os.path.exists(pwo.REF_FAST_BIN):
        pytest.skip("reference not built (make -C oracle ref)")
    tmp = tempfile.mkdtemp()
    toks, lens, comm = synth.dcsbm_walks(seed=2)
    corpus = os.path.join(tmp, "walks.txt")
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
    counts = vocab.counts()
    labels = np.array([comm[int(w[1:])] if w.startswith(b"w") else -1 for w in vocab.words()], np.int64)
    queries = np.flatnonzero(labels >= 0)
    triples = evaluate.eval_triples(stream, counts, n_windows=4096, window=10)
    run = dict(V=V, d=d, stream=stream, counts=counts, labels=labels, queries=queries, triples=triples)
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
    return loss, evaluate.recall_at_10(w_in, run["labels"], run["queries"], device="cuda")


@pytest.mark.parametrize("mode,variant", [(pw.MODE_PLAIN, 0), (pw.MODE_BATCHED, pw.VARIANT_STREAM),
                                          (pw.MODE_BATCHED_BF16, pw.VARIANT_WINDOW),
                                          (pw.MODE_BATCHED_BF16, pw.VARIANT_STREAM)])
def test_graph_matches_reference_loss_and_recall(graph_run, mode, variant):
    run = graph_run
    ref_loss, ref_rec = run["ref_loss"], run["ref_recall"]
    with pw.Trainer(mode=mode, seed=1, variant=variant, size=FLAGS["size"], window=FLAGS["window"],
                    negative=FLAGS["negative"], batch_size=FLAGS["batch_size"], iter=FLAGS["iter"],
                    alpha=float(FLAGS["alpha"]), sample=0.0) as t:
        t.set_vocab(run["counts"])
        t.init_weights()
        t.set_corpus(run["stream"])
        st = t.train()
        w_in, w_out = t.get_weights()
    assert np.isfinite(w_in).all() and np.isfinite(w_out).all()
    assert st["words"] == len(run["stream"])
    assert st["kept"] == int((run["stream"] != 0).sum())  # no subsampling: every node visit trains
    # window 10 draws up to 19 * 5 = 95 shared negatives per batch: the BATCHED modes still take
    # the tensor-core repulsion
    want = pw.REPULSION_SERIAL if mode == pw.MODE_PLAIN else pw.REPULSION_TENSOR
    assert st["repulsion"] == want
    loss, rec = score(run, w_in, w_out)
    print(f"graph mode {mode} variant {variant}: loss {loss:.5f} (ref mean {ref_loss:.5f} of {run['ref_losses']}) recall {rec:.4f} "
          f"(ref {ref_rec:.4f}) ms {st['kernel_ms']:.1f}")
    assert abs(loss - ref_loss) <= 0.01 * ref_loss
    assert abs(rec - ref_rec) <= 0.01
