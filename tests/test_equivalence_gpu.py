"""With one warp in flight the Hogwild modes are sequential: PLAIN and BATCHED then make the
same random decisions (same LCG stream per sentence, same draw order) and must produce the same
weights up to floating-point summation order.  This pins the data-local kernel's bookkeeping
(window ring, duplicate-word ownership, prefetch, chunked repulsion, merged write-back) to the
straightforward kernel, independently of Hogwild effects."""
import numpy as np
import pytest

import par_word2vec_b200 as pw

pytestmark = pytest.mark.gpu


def run(golden, mode, attraction=pw.ATTRACT_SEQUENTIAL, variant=pw.VARIANT_AUTO, **over):
    k = golden.train_kwargs()
    k.update(over)
    with pw.Trainer(mode=mode, seed=3, grid=1, warps_per_cta=1, attraction=attraction, variant=variant, **k) as t:
        t.set_vocab(golden.counts)
        t.init_weights()
        t.set_corpus(golden.stream[:-1])
        st = t.train()
        return st, t.get_weights()


@pytest.mark.parametrize("variant", [pw.VARIANT_WINDOW, pw.VARIANT_STREAM])
@pytest.mark.parametrize("attraction", [pw.ATTRACT_SEQUENTIAL, pw.ATTRACT_WINDOW, pw.ATTRACT_PIPELINED])
@pytest.mark.parametrize("case", ["text_small", "graph_small", "edge", "d100"])
def test_batched_fp32_equals_plain_sequentially(golden_cases, case, attraction, variant):
    """PIPELINED (streamed kernel) computes SEQUENTIAL's updates: PLAIN, which runs SEQUENTIAL
    for it, is the reference for both."""
    g = golden_cases[case]
    sp, (pi, po) = run(g, pw.MODE_PLAIN, attraction)
    sb, (bi, bo) = run(g, pw.MODE_BATCHED, attraction, variant)
    for k in ("kept", "sentences", "pairs", "batches", "negatives"):
        assert sp[k] == sb[k], k
    scale = max(np.abs(pi).max(), np.abs(po).max())
    err_in = np.abs(pi - bi).max() / scale
    err_out = np.abs(po - bo).max() / scale
    print(case, "max rel diff W_in", err_in, "W_out", err_out)
    assert err_in < 1e-4 and err_out < 1e-4


@pytest.mark.parametrize("variant", [pw.VARIANT_WINDOW, pw.VARIANT_STREAM])
@pytest.mark.parametrize("attraction", [pw.ATTRACT_SEQUENTIAL, pw.ATTRACT_WINDOW, pw.ATTRACT_PIPELINED])
@pytest.mark.parametrize("case", ["text_small", "d100"])
def test_batched_bf16_tracks_plain_sequentially(golden_cases, case, attraction, variant):
    """BF16 tables with stochastic rounding (and, for these shapes, the tensor-core repulsion)
    stay within a few percent of the FP32 run that makes the same random decisions."""
    g = golden_cases[case]
    _, (pi, po) = run(g, pw.MODE_PLAIN, attraction)
    _, (bi, bo) = run(g, pw.MODE_BATCHED_BF16, attraction, variant)
    rel = np.linalg.norm(bi - pi) / np.linalg.norm(pi)
    print(case, "BF16 relative Frobenius error of W_in", rel)
    assert rel < 0.05
