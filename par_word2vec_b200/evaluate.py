"""Embedding-quality measures used to compare training modes with the reference.

* ``recall_at_10``  -- planted-cluster recall@10: for each query word, the fraction of its 10
  cosine-nearest neighbours in W_in (excluding itself and "</s>") that carry the query's
  planted label.  Chance level is 1 / number of labels.
* ``topic_margin`` -- cosine to the query's planted-topic centroid minus the mean cosine to the
  other centroids: continuous, where recall@10 of these corpora saturates near 1.
* ``eval_triples`` / ``sgns_loss`` -- a fixed, seeded evaluation set of (target, context,
  negatives) windows drawn from a corpus, scored with the library's FP64 loss kernel.

These are measurements, not part of the training path; they run with numpy (or torch on the
GPU when available, for the 555k-word vocabularies of the 1B-word-shaped corpus).
"""
from __future__ import annotations

import numpy as np


def labels_from_words(words: list[bytes], n_labels: int, prefix: bytes = b"w") -> np.ndarray:
    """Planted label of each vocabulary row (generator id modulo n_labels; -1 for "</s>")."""
    out = np.full(len(words), -1, dtype=np.int64)
    for i, w in enumerate(words):
        if w.startswith(prefix) and w[len(prefix):].isdigit():
            out[i] = int(w[len(prefix):]) % n_labels
    return out


def recall_at_10(w_in: np.ndarray, labels: np.ndarray, queries: np.ndarray, k: int = 10,
                 device: str | None = None) -> float:
    """Mean fraction of the k nearest neighbours (cosine) sharing the query's label."""
    valid = labels >= 0
    try:
        import torch
        use_torch = device is not None and torch.cuda.is_available()
    except Exception:
        use_torch = False
    if use_torch:
        import torch
        W = torch.from_numpy(np.ascontiguousarray(w_in, np.float32)).to(device)
        W = W / W.norm(dim=1, keepdim=True).clamp_min(1e-12)
        lab = torch.from_numpy(labels).to(device)
        bad = torch.from_numpy(~valid).to(device)
        hits = 0.0
        for s in range(0, len(queries), 2048):
            q = torch.from_numpy(queries[s: s + 2048].astype(np.int64)).to(device)
            sim = W[q] @ W.T
            sim[:, bad] = -np.inf
            sim[torch.arange(len(q), device=device), q] = -np.inf
            nn = sim.topk(k, dim=1).indices
            hits += (lab[nn] == lab[q][:, None]).float().sum().item()
        return hits / (len(queries) * k)
    W = np.asarray(w_in, np.float32)
    W = W / np.maximum(np.linalg.norm(W, axis=1, keepdims=True), 1e-12)
    hits = 0
    for s in range(0, len(queries), 512):
        q = queries[s: s + 512]
        sim = W[q] @ W.T
        sim[:, ~valid] = -np.inf
        sim[np.arange(len(q)), q] = -np.inf
        nn = np.argpartition(-sim, k, axis=1)[:, :k]
        hits += int((labels[nn] == labels[q][:, None]).sum())
    return hits / (len(queries) * k)


def topic_margin(w_in: np.ndarray, labels: np.ndarray, queries: np.ndarray, device: str | None = None) -> float:
    """A continuous measure of the planted structure that does not saturate like recall@10: the
    mean over the queries of cos(q, own topic's centroid) minus the mean cos(q, other topics'
    centroids), with centroids the normalised means of the unit vectors of all labelled words."""
    valid = labels >= 0
    n_lab = int(labels.max()) + 1
    try:
        import torch
        use_torch = device is not None and torch.cuda.is_available()
    except Exception:
        use_torch = False
    if use_torch:
        import torch
        W = torch.from_numpy(np.ascontiguousarray(w_in, np.float32)).to(device)
        W = W / W.norm(dim=1, keepdim=True).clamp_min(1e-12)
        lab = torch.from_numpy(labels).to(device)
        idx = torch.from_numpy(np.flatnonzero(valid)).to(device)
        C = torch.zeros(n_lab, W.shape[1], device=device).index_add_(0, lab[idx], W[idx])
        C = C / C.norm(dim=1, keepdim=True).clamp_min(1e-12)
        q = torch.from_numpy(queries.astype(np.int64)).to(device)
        S = W[q] @ C.T
        own = S.gather(1, lab[q][:, None]).squeeze(1)
        other = (S.sum(dim=1) - own) / (n_lab - 1)
        return float((own - other).mean().item())
    W = np.asarray(w_in, np.float32)
    W = W / np.maximum(np.linalg.norm(W, axis=1, keepdims=True), 1e-12)
    C = np.zeros((n_lab, W.shape[1]), np.float64)
    np.add.at(C, labels[valid], W[valid])
    C /= np.maximum(np.linalg.norm(C, axis=1, keepdims=True), 1e-12)
    S = W[queries] @ C.T
    own = S[np.arange(len(queries)), labels[queries]]
    other = (S.sum(axis=1) - own) / (n_lab - 1)
    return float((own - other).mean())


def top_queries(counts: np.ndarray, labels: np.ndarray, n: int) -> np.ndarray:
    """The n most frequent labelled words (vocabulary rows are sorted by count already)."""
    idx = np.flatnonzero(labels >= 0)
    order = idx[np.argsort(-counts[idx].astype(np.int64), kind="stable")]
    return order[:n].astype(np.int64)


def eval_triples(stream: np.ndarray, counts: np.ndarray, n_windows: int = 4096, window: int = 5,
                 ctx_per_window: int = 10, n_neg: int = 15, seed: int = 7):
    """Seeded (target, context) windows from the corpus with negatives drawn from unigram^0.75."""
    rng = np.random.default_rng(seed)
    s = np.asarray(stream)
    n = len(s)
    p = counts.astype(np.float64) ** 0.75
    p[0] = 0.0
    p /= p.sum()
    tgt, ctx, neg = [], [], []
    while len(tgt) < n_windows:
        i = int(rng.integers(window, n - window))
        t = int(s[i])
        if t == 0:
            continue
        around = s[i - window: i + window + 1]
        c = [int(x) for j, x in enumerate(around) if j != window and x != 0]
        if len(c) < 2:
            continue
        c = (c * ctx_per_window)[:ctx_per_window]
        tgt.append([t] * ctx_per_window)
        ctx.append(c)
        neg.append(rng.choice(len(p), size=n_neg, p=p))
    return (np.array(tgt, np.int32).ravel(), np.array(ctx, np.int32).ravel(), np.array(neg, np.int32).ravel())


def sgns_loss(trainer, triples, n_neg: int = 15, ctx_per_window: int = 10) -> float:
    """Mean SGNS loss per (target, context) pair of the evaluation set, FP64 reduction on the GPU."""
    tgt, ctx, neg = triples
    return trainer.loss(tgt, ctx, neg, n_neg, ctx_per_window) / len(tgt)
