"""SGNS loss, its hand-written adjoint and FP64 central finite differences on the device.

Workload (the adjoint check): vocabulary 100,000, d = 300, W_in ~ U(-0.5/d, 0.5/d),
W_out ~ N(0, 0.1); 4,096 (target, context) pairs drawn from Zipf(1.0); windows of 10 contexts
share 15 negatives drawn from the unigram^0.75 table (410 windows, the last one ragged).

Checked, in FP32 and in BF16 tables:
  * parw2v_loss against a float64 numpy evaluation of the same sum;
  * parw2v_loss_adjoint(exact=1) against FP64 central differences (h = 1e-3) at probes on every
    kind of touched row (contexts in W_in, targets and negatives in W_out), and against the float64
    numpy gradient over the whole matrices;
  * parw2v_loss_adjoint(exact=0) against the reference's update rule restated in numpy: the
    expTable sigma with the +-6 clamp, g = label - sigma (PAR_Word2Vec_cpu.cpp:554-559, :642-647),
    i.e. the reference's attraction and repulsion updates divided by -alpha.
BF16: the adjoint on BF16-stored weights is exact arithmetic on those weights (same tolerance as
FP32 against FD on the stored values); its error against the FP64 gradient at the original FP32
weights is the storage error, stated here and bounded by 1%."""
import numpy as np
import pytest

import par_word2vec_b200 as pw

pytestmark = pytest.mark.gpu

V, D, PAIRS, CPW, NNEG = 100_000, 300, 4096, 10, 15


@pytest.fixture(scope="module")
def batch():
    rng = np.random.default_rng(3)
    w_in = rng.uniform(-0.5 / D, 0.5 / D, size=(V, D)).astype(np.float32)
    w_out = rng.normal(0.0, 0.1, size=(V, D)).astype(np.float32)
    ranks = np.arange(1, V, dtype=np.float64)
    p = 1.0 / ranks
    p /= p.sum()
    tgt = (rng.choice(V - 1, size=PAIRS, p=p) + 1).astype(np.int32)
    ctx = (rng.choice(V - 1, size=PAIRS, p=p) + 1).astype(np.int32)
    counts = (1e7 / np.arange(1, V + 1)).astype(np.uint32) + 1
    return dict(rng=rng, w_in=w_in, w_out=w_out, tgt=tgt, ctx=ctx, counts=counts)


def negatives(trainer, b):
    table = trainer.get_table()
    n_win = (PAIRS + CPW - 1) // CPW
    idx = b["rng"].integers(0, len(table), size=n_win * NNEG)
    neg = table[idx].astype(np.int32)
    zero = neg == 0  # the reference redraws a 0 uniformly (PAR_Word2Vec_cpu.cpp:605-606)
    neg[zero] = b["rng"].integers(1, V, size=int(zero.sum()))
    return neg


def sigma(x):
    return 1.0 / (1.0 + np.exp(-x))


def fp64_terms(w_in, w_out, tgt, ctx, neg):
    u = w_in[ctx].astype(np.float64)
    v = w_out[tgt].astype(np.float64)
    win = np.arange(PAIRS) // CPW
    nk = neg.reshape(-1, NNEG)[win]               # PAIRS x NNEG negative ids
    vk = w_out[nk].astype(np.float64)             # PAIRS x NNEG x D
    f = (u * v).sum(1)
    fk = np.einsum("pd,pkd->pk", u, vk)
    return u, v, nk, vk, f, fk


def fp64_loss(w_in, w_out, tgt, ctx, neg):
    _, _, _, _, f, fk = fp64_terms(w_in, w_out, tgt, ctx, neg)
    return np.logaddexp(0, -f).sum() + np.logaddexp(0, fk).sum()


def fp64_grad(w_in, w_out, tgt, ctx, neg, df=None, dfk=None):
    """dL/dW_in, dL/dW_out given dL/df per pair and dL/df_k per (pair, negative)."""
    u, v, nk, vk, f, fk = fp64_terms(w_in, w_out, tgt, ctx, neg)
    if df is None:
        df, dfk = sigma(f) - 1.0, sigma(fk)
    else:
        df, dfk = df(f), dfk(fk)
    g_in = np.zeros((V, D))
    g_out = np.zeros((V, D))
    np.add.at(g_in, ctx, df[:, None] * v + np.einsum("pk,pkd->pd", dfk, vk))
    np.add.at(g_out, tgt, df[:, None] * u)
    np.add.at(g_out, nk.ravel(), (dfk[:, :, None] * u[:, None, :]).reshape(-1, D))
    return g_in, g_out


def table_sigma(exp, label):
    """The reference's sigma for a label's update: expTable index (f + 6) * 1000/12, clamped at +-6."""
    def s(f):
        f32 = f.astype(np.float32)
        idx = np.floor((f32 + np.float32(6)) * np.float32(1000.0 / 12.0)).astype(np.int64)
        out = exp[np.clip(idx, 0, 1000)].astype(np.float64)
        out[f32 > 6] = 1.0
        out[f32 < -6] = 0.0
        return out - label
    return s


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def probes(b, neg, n=96):
    rng = np.random.default_rng(5)
    rows_in = rng.choice(b["ctx"], size=n)
    rows_t = rng.choice(b["tgt"], size=n // 2)
    rows_n = rng.choice(neg, size=n - n // 2)
    matrix = np.concatenate([np.zeros(n, np.int32), np.ones(n, np.int32)])
    row = np.concatenate([rows_in, rows_t, rows_n]).astype(np.int32)
    col = rng.integers(0, D, size=2 * n).astype(np.int32)
    return matrix, row, col


@pytest.mark.parametrize("mode", [pw.MODE_PLAIN, pw.MODE_BATCHED_BF16])
def test_adjoint_against_fp64_finite_differences(batch, mode):
    b = batch
    with pw.Trainer(mode=mode, size=D) as t:
        t.set_vocab(b["counts"])
        neg = negatives(t, b)
        t.set_weights(b["w_in"], b["w_out"])
        w_in, w_out = t.get_weights()  # the stored weights (BF16 widened in BF16 mode)
        loss = t.loss(b["tgt"], b["ctx"], neg, NNEG, CPW)
        g_in, g_out = t.loss_adjoint(b["tgt"], b["ctx"], neg, NNEG, CPW, exact=True)
        matrix, row, col = probes(b, neg)
        fd = t.loss_fd(b["tgt"], b["ctx"], neg, NNEG, CPW, matrix, row, col, h=1e-3)
    want_loss = fp64_loss(w_in, w_out, b["tgt"], b["ctx"], neg)
    assert abs(loss - want_loss) <= 1e-6 * abs(want_loss)
    adj = np.where(matrix == 0, g_in[row, col], g_out[row, col]).astype(np.float64)
    err_fd = rel(adj, fd)
    ref_in, ref_out = fp64_grad(w_in, w_out, b["tgt"], b["ctx"], neg)
    err_in, err_out = rel(g_in, ref_in), rel(g_out, ref_out)
    print(f"mode {mode}: loss {loss:.6f}; "
          f"adjoint vs FD rel {err_fd:.2e}; vs FP64 gradient W_in {err_in:.2e} W_out {err_out:.2e}")
    assert err_fd < 1e-4
    assert np.abs(adj - fd).max() <= 1e-4 * np.abs(fd).max() + 1e-6
    assert err_in < 1e-5 and err_out < 1e-5


def test_reference_rule_adjoint(batch):
    b = batch
    with pw.Trainer(mode=pw.MODE_PLAIN, size=D) as t:
        t.set_vocab(b["counts"])
        neg = negatives(t, b)
        exp = t.get_exp_table()
        t.set_weights(b["w_in"], b["w_out"])
        r_in, r_out = t.loss_adjoint(b["tgt"], b["ctx"], neg, NNEG, CPW, exact=False)
        e_in, e_out = t.loss_adjoint(b["tgt"], b["ctx"], neg, NNEG, CPW, exact=True)
    want_in, want_out = fp64_grad(b["w_in"], b["w_out"], b["tgt"], b["ctx"], neg,
                                  df=table_sigma(exp, 1.0), dfk=table_sigma(exp, 0.0))
    err_in, err_out = rel(r_in, want_in), rel(r_out, want_out)
    # the table's step in f is 12/1000, so its sigma differs from the exact one by < 0.003
    gap_in, gap_out = rel(r_in, e_in), rel(r_out, e_out)
    print(f"reference rule vs numpy rule: W_in {err_in:.2e} W_out {err_out:.2e}; "
          f"rule vs exact adjoint: W_in {gap_in:.2e} W_out {gap_out:.2e}")
    assert err_in < 1e-4 and err_out < 1e-4
    assert gap_in < 0.01 and gap_out < 0.01


def test_bf16_storage_error_against_fp64(batch):
    """The gradient computed from BF16-stored weights, against the FP64 gradient at the FP32
    weights the caller set: the error BF16 storage costs one step."""
    b = batch
    with pw.Trainer(mode=pw.MODE_BATCHED_BF16, size=D) as t:
        t.set_vocab(b["counts"])
        neg = negatives(t, b)
        t.set_weights(b["w_in"], b["w_out"])
        g_in, g_out = t.loss_adjoint(b["tgt"], b["ctx"], neg, NNEG, CPW, exact=True)
        s_in, s_out = t.get_weights()
    ref_in, ref_out = fp64_grad(b["w_in"], b["w_out"], b["tgt"], b["ctx"], neg)
    err_in, err_out = rel(g_in, ref_in), rel(g_out, ref_out)
    w_err = max(rel(s_in, b["w_in"]), rel(s_out, b["w_out"]))
    print(f"BF16: weight storage rel err {w_err:.2e}; gradient vs FP64 at the FP32 weights: "
          f"W_in {err_in:.2e} W_out {err_out:.2e}")
    assert w_err < 2.0 ** -8
    assert err_in < 0.01 and err_out < 0.01
