"""The unigram^0.75 table at full vocabulary sizes (the 1B-shaped bench's ~555k words and the
text8-shaped 71k), built on the device: a warp-fed FP64 total and float running sum in the
reference's order, parallel quotients and threshold searches, slot starts as a prefix maximum,
a parallel fill.  The bar is byte equality with the oracle's restatement of the reference's
one-slot-at-a-time loop (PAR_Word2Vec_cpu.cpp:96-117, one thread)."""
import numpy as np
import pytest

import par_word2vec_b200 as pw
from oracle import pwo

pytestmark = pytest.mark.gpu


def zipf_counts(V: int, seed: int) -> np.ndarray:
    """Descending Zipf-like counts with ties and a min-count floor, as a sorted vocabulary has."""
    rng = np.random.default_rng(seed)
    c = 4e8 / np.arange(1, V + 1) * rng.uniform(0.97, 1.03, V)
    return np.sort(np.maximum(c, 5).astype(np.uint32))[::-1].copy()


@pytest.mark.parametrize("V", [555_001, 71_291])
def test_table_matches_reference_loop(V):
    counts = zipf_counts(V, V)
    with pw.Trainer(size=16, mode=pw.MODE_PLAIN) as t:
        t.set_vocab(counts)
        got = t.get_table()
    want = pwo.unigram_table(counts)
    assert got.shape == want.shape
    bad = np.flatnonzero(got != want)
    assert bad.size == 0, f"{bad.size} slots differ, first at {bad[0]}: {got[bad[0]]} vs {want[bad[0]]}"
    assert got[0] == 0
