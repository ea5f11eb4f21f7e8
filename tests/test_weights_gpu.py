"""Weight transfer through the C ABI (parw2v_set_weights / parw2v_get_weights).

The device keeps rows of ld >= d elements (FP32, or BF16 in the BF16 mode) and the host rows of d
FP32 values; the transfer runs through a staging buffer of at most 64 MiB of dense rows, one
row-layout kernel and one linear copy per chunk.  Checked: FP32 tables return exactly what was
set; BF16 tables return the round-to-nearest-even BF16 value of what was set; d not a multiple of
4 (padded device rows), a table spanning several staging chunks, a two-row table, and one-sided
reads."""
import numpy as np
import pytest

import par_word2vec_b200 as pw

pytestmark = pytest.mark.gpu


def bf16_rne(x: np.ndarray) -> np.ndarray:
    """FP32 -> BF16 -> FP32 with round-to-nearest-even, for finite values."""
    u = x.astype(np.float32).view(np.uint32).astype(np.uint64)
    r = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return r.astype(np.uint32).view(np.float32)


@pytest.mark.parametrize("mode", [pw.MODE_PLAIN, pw.MODE_BATCHED, pw.MODE_BATCHED_BF16])
@pytest.mark.parametrize("V,d", [(2, 1), (1000, 301), (120_001, 300)])
def test_set_get_round_trip(mode, V, d):
    # (120,001 x 300) FP32 rows are 137 MB: three staging chunks, the last one partial
    rng = np.random.default_rng(V + d)
    w_in = rng.standard_normal((V, d)).astype(np.float32)
    w_out = rng.standard_normal((V, d)).astype(np.float32)
    with pw.Trainer(mode=mode, size=d) as t:
        t.set_vocab(np.full(V, 10, np.uint32))
        t.set_weights(w_in, w_out)
        got_in, got_out = t.get_weights()
        only_out = t.get_weights("out")
    if mode == pw.MODE_BATCHED_BF16:
        w_in, w_out = bf16_rne(w_in), bf16_rne(w_out)
    assert np.array_equal(got_in, w_in)
    assert np.array_equal(got_out, w_out)
    assert np.array_equal(only_out, w_out)


def test_partial_update_keeps_the_other_table():
    V, d = 5000, 130
    rng = np.random.default_rng(9)
    a, b, c = (rng.standard_normal((V, d)).astype(np.float32) for _ in range(3))
    with pw.Trainer(mode=pw.MODE_PLAIN, size=d) as t:
        t.set_vocab(np.full(V, 10, np.uint32))
        t.set_weights(a, b)
        t.set_weights(w_in=c)
        got_in, got_out = t.get_weights()
    assert np.array_equal(got_in, c)
    assert np.array_equal(got_out, b)
