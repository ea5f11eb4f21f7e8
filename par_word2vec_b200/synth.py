"""Seeded synthetic corpora that stand in for the reference's public datasets.

The reference trains on text8, the 1B-word benchmark and random walks over five social
graphs (``data.sh``, ``SC19_AE_test_cases/Table*.sh``).  None of those datasets is
available here, so these generators produce corpora with the same shapes and a
*planted* structure that embedding quality can be scored against:

* ``topic_zipf``   -- documents of word ids.  Each document picks one of ``n_topics``
  latent topics; each token is drawn with probability ``p_global`` from a global
  Zipf(s) over all ids, else from a Zipf(s) over the topic's slice
  ``{id : id % n_topics == topic}``.  The planted label of word id ``i`` is
  ``i % n_topics``.  text8-shaped: 17,000 documents x 1,000 tokens over 71,290 ids,
  64 topics.  1B-word-shaped: lognormal sentence lengths (mean 25, sigma 1.0,
  clipped to 1..1000), 256 topics.
* ``dcsbm_walks``  -- a degree-corrected stochastic block model graph and uniform
  random walks over it (10 walks of length 80 per node).  The planted label of a
  node is its community.

Tokens are written as ``w<id>`` (``n<id>`` for nodes), one document / walk per line,
so every line ends with the reference's "</s>" token (``ReadWord``,
PAR_Word2Vec_cpu.cpp:119-144).
"""
from __future__ import annotations

import numpy as np


def _zipf_cdf(n: int, s: float) -> np.ndarray:
    p = 1.0 / np.arange(1, n + 1, dtype=np.float64) ** s
    c = np.cumsum(p)
    return c / c[-1]


def _draw(cdf: np.ndarray, u: np.ndarray) -> np.ndarray:
    return np.minimum(np.searchsorted(cdf, u, side="right"), len(cdf) - 1)


def topic_zipf(n_tokens_or_docs, n_types: int, n_topics: int, *, doc_len: int | None = 1000,
               lognormal_mean: float | None = None, lognormal_sigma: float = 1.0,
               p_global: float = 0.5, s: float = 1.0, seed: int = 1):
    """Return ``(tokens, lengths)``: int32 generator ids and per-document lengths.

    With ``doc_len`` set, ``n_tokens_or_docs`` is the number of documents of that
    length.  With ``lognormal_mean`` set, lengths are lognormal with that mean and
    ``lognormal_sigma``, clipped to 1..1000, until ``n_tokens_or_docs`` tokens.
    """
    rng = np.random.default_rng(seed)
    if lognormal_mean is not None:
        n_tokens = int(n_tokens_or_docs)
        mu = np.log(lognormal_mean) - 0.5 * lognormal_sigma ** 2
        est = int(n_tokens / lognormal_mean * 1.2) + 16
        lengths = np.clip(np.rint(rng.lognormal(mu, lognormal_sigma, est)), 1, 1000).astype(np.int64)
        csum = np.cumsum(lengths)
        while csum[-1] < n_tokens:
            more = np.clip(np.rint(rng.lognormal(mu, lognormal_sigma, est)), 1, 1000).astype(np.int64)
            lengths = np.concatenate([lengths, more])
            csum = np.cumsum(lengths)
        k = int(np.searchsorted(csum, n_tokens))
        lengths = lengths[: k + 1].copy()
        lengths[-1] -= int(csum[k] - n_tokens)
        lengths = lengths[lengths > 0]
    else:
        lengths = np.full(int(n_tokens_or_docs), int(doc_len), dtype=np.int64)
    n = int(lengths.sum())
    n_docs = len(lengths)
    topic_of_doc = rng.integers(0, n_topics, n_docs)
    topic = np.repeat(topic_of_doc, lengths)
    slice_len = -(-n_types // n_topics)
    g_cdf = _zipf_cdf(n_types, s)
    l_cdf = _zipf_cdf(slice_len, s)
    use_global = rng.random(n) < p_global
    out = np.empty(n, dtype=np.int64)
    ng = int(use_global.sum())
    out[use_global] = _draw(g_cdf, rng.random(ng))
    loc = ~use_global
    r = _draw(l_cdf, rng.random(n - ng))
    ids = topic[loc] + n_topics * r
    # slices at the top end are one id shorter when n_types % n_topics != 0
    over = ids >= n_types
    ids[over] = topic[loc][over]
    out[loc] = ids
    return out.astype(np.int32), lengths


def dcsbm_walks(n_nodes: int = 10312, n_comm: int = 39, n_edges: int = 334000, *,
                intra: float = 0.7, exponent: float = 2.5, walks_per_node: int = 10,
                walk_len: int = 80, seed: int = 2):
    """Return ``(tokens, lengths, community)`` for uniform random walks on a DC-SBM graph."""
    rng = np.random.default_rng(seed)
    comm = rng.integers(0, n_comm, n_nodes)
    theta = (1.0 - rng.random(n_nodes)) ** (-1.0 / (exponent - 1.0))  # Pareto, x_min = 1
    members = [np.flatnonzero(comm == c) for c in range(n_comm)]
    cdfs = []
    for m in members:
        w = np.cumsum(theta[m])
        cdfs.append(w / w[-1] if len(m) else w)
    g = np.cumsum(theta)
    g /= g[-1]
    comm_mass = np.array([theta[m].sum() for m in members])
    comm_cdf = np.cumsum(comm_mass) / comm_mass.sum()
    edges = set()
    target = int(n_edges)
    while len(edges) < target:
        batch = max(1024, int((target - len(edges)) * 1.3))
        is_in = rng.random(batch) < intra
        u = np.empty(batch, dtype=np.int64)
        v = np.empty(batch, dtype=np.int64)
        cs = _draw(comm_cdf, rng.random(batch))
        for c in np.unique(cs[is_in]):
            sel = np.flatnonzero(is_in & (cs == c))
            m = members[c]
            u[sel] = m[_draw(cdfs[c], rng.random(len(sel)))]
            v[sel] = m[_draw(cdfs[c], rng.random(len(sel)))]
        sel = np.flatnonzero(~is_in)
        u[sel] = _draw(g, rng.random(len(sel)))
        v[sel] = _draw(g, rng.random(len(sel)))
        ok = (u != v) & ((comm[u] == comm[v]) == is_in)
        for a, b in zip(u[ok].tolist(), v[ok].tolist()):
            if len(edges) >= target:
                break
            edges.add((a, b) if a < b else (b, a))
    e = np.array(sorted(edges), dtype=np.int64)
    deg = np.bincount(e.ravel(), minlength=n_nodes)
    # every node gets at least one neighbour in its own community so that walks can move
    lonely = np.flatnonzero(deg == 0)
    extra = []
    for x in lonely.tolist():
        m = members[comm[x]]
        y = int(m[rng.integers(0, len(m))]) if len(m) > 1 else int(rng.integers(0, n_nodes))
        if y == x:
            y = (x + 1) % n_nodes
        extra.append((min(x, y), max(x, y)))
    if extra:
        e = np.concatenate([e, np.array(extra, dtype=np.int64)])
    src = np.concatenate([e[:, 0], e[:, 1]])
    dst = np.concatenate([e[:, 1], e[:, 0]])
    order = np.argsort(src, kind="stable")
    src, dst = src[order], dst[order]
    indptr = np.zeros(n_nodes + 1, dtype=np.int64)
    np.add.at(indptr, src + 1, 1)
    indptr = np.cumsum(indptr)
    starts = np.tile(np.arange(n_nodes, dtype=np.int64), walks_per_node)
    walks = np.empty((len(starts), walk_len), dtype=np.int64)
    cur = starts
    walks[:, 0] = cur
    for step in range(1, walk_len):
        deg_c = indptr[cur + 1] - indptr[cur]
        pick = indptr[cur] + (rng.random(len(cur)) * deg_c).astype(np.int64)
        cur = dst[pick]
        walks[:, step] = cur
    lengths = np.full(len(starts), walk_len, dtype=np.int64)
    return walks.ravel().astype(np.int32), lengths, comm.astype(np.int32)


def write_text(path: str, tokens: np.ndarray, lengths: np.ndarray, prefix: str = "w") -> int:
    """Write one document per line as ``<prefix><id>`` tokens; returns bytes written."""
    names = np.array([f"{prefix}{i}" for i in range(int(tokens.max()) + 1)], dtype=object)
    off = 0
    total = 0
    with open(path, "w") as f:
        chunk = []
        for ln in lengths.tolist():
            chunk.append(" ".join(names[tokens[off: off + ln]].tolist()))
            off += ln
            if len(chunk) >= 4096:
                s = "\n".join(chunk) + "\n"
                f.write(s)
                total += len(s)
                chunk = []
        if chunk:
            s = "\n".join(chunk) + "\n"
            f.write(s)
            total += len(s)
    return total


def write_stream_text(path: str, stream: np.ndarray, words: list[bytes], chunk: int = 1 << 23) -> int:
    """Write a vocabulary-id stream (0 = "</s>" ends a line) as reference-readable text: every
    word followed by a space, a newline per "</s>" (the reference's tokenizer reads the same ids
    back, PAR_Word2Vec_cpu.cpp:120-144).  Vectorised over chunks of
    the stream (a gather of the words' bytes), so 10^8 tokens take seconds.  Returns bytes written."""
    lens = np.array([len(w) + 1 for w in words], dtype=np.int64)  # word + separator
    lens[0] = 1  # "</s>" is written as the newline alone
    flat = np.frombuffer(b"".join([b"\n"] + [w + b" " for w in words[1:]]), dtype=np.uint8)
    starts = np.concatenate([[0], np.cumsum(lens)[:-1]])
    s = np.asarray(stream)
    total = 0
    with open(path, "wb") as f:
        for c0 in range(0, len(s), chunk):
            ids = s[c0: c0 + chunk].astype(np.int64)
            ln = lens[ids]
            out_start = np.cumsum(ln) - ln
            src = np.repeat(starts[ids] - out_start, ln) + np.arange(int(ln.sum()), dtype=np.int64)
            buf = flat[src]  # each word keeps its trailing space, also before a newline
            f.write(buf.tobytes())
            total += len(buf)
    return total


def topic_zipf_stream_torch(n_tokens: int, n_types: int, n_topics: int, *, lognormal_mean: float = 25.0,
                            lognormal_sigma: float = 1.0, p_global: float = 0.5, s: float = 1.0, seed: int = 4,
                            min_count: int = 5, device: str = "cuda"):
    """The 1B-word-shaped corpus built directly as a vocabulary-id stream on the GPU.

    Same generator as ``topic_zipf`` with lognormal sentence lengths; the vocabulary step is
    the reference's (counts, "</s>" first, descending count, min_count filter), with ties in
    count ordered by generator id (the text path orders ties as the reference's qsort does).
    Returns ``(stream_int32_device, counts_uint32_numpy, words_list, gen_ids_of_rows)`` where
    the stream holds one 0 ("</s>") after every sentence.
    """
    import torch

    g = torch.Generator(device=device)
    g.manual_seed(seed)
    mu = float(np.log(lognormal_mean) - 0.5 * lognormal_sigma ** 2)
    est = int(n_tokens / lognormal_mean * 1.1) + 1024
    lengths = torch.empty(0, dtype=torch.int64, device=device)
    while int(lengths.sum()) < n_tokens:
        more = torch.empty(est, device=device, dtype=torch.float64).log_normal_(mu, lognormal_sigma, generator=g)
        lengths = torch.cat([lengths, more.round().clamp_(1, 1000).to(torch.int64)])
    csum = torch.cumsum(lengths, 0)
    k = int(torch.searchsorted(csum, torch.tensor([n_tokens], device=device)).item())
    lengths = lengths[: k + 1].clone()
    lengths[-1] -= int(csum[k].item()) - n_tokens
    lengths = lengths[lengths > 0]
    n_sent = len(lengths)
    topic = torch.randint(0, n_topics, (n_sent,), generator=g, device=device)
    g_cdf = torch.from_numpy(_zipf_cdf(n_types, s)).to(device)
    slice_len = -(-n_types // n_topics)
    l_cdf = torch.from_numpy(_zipf_cdf(slice_len, s)).to(device)
    ids = torch.empty(n_tokens, dtype=torch.int64, device=device)
    chunk = 1 << 27
    tok_topic_all = torch.repeat_interleave(topic, lengths)
    for s0 in range(0, n_tokens, chunk):
        s1 = min(n_tokens, s0 + chunk)
        m = s1 - s0
        u = torch.rand(m, generator=g, device=device, dtype=torch.float64)
        use_g = torch.rand(m, generator=g, device=device) < p_global
        gi = torch.searchsorted(g_cdf, u, right=True).clamp_(max=n_types - 1)
        li = torch.searchsorted(l_cdf, u, right=True).clamp_(max=slice_len - 1)
        tt = tok_topic_all[s0:s1]
        loc = tt + n_topics * li
        loc = torch.where(loc >= n_types, tt, loc)
        ids[s0:s1] = torch.where(use_g, gi, loc)
    del tok_topic_all
    cnt = torch.bincount(ids, minlength=n_types)
    # vocabulary order: descending count, ties by generator id; "</s>" is row 0
    order = torch.argsort(-cnt * (n_types + 1) + torch.arange(n_types, device=device))
    cnt_sorted = cnt[order]
    keep = cnt_sorted >= min_count
    order = order[keep]
    row_of = torch.full((n_types,), -1, dtype=torch.int64, device=device)
    row_of[order] = torch.arange(1, len(order) + 1, device=device)
    rows = row_of[ids]
    del ids
    # stream: sentence tokens followed by a 0, dropping filtered (-1) words
    ends = torch.cumsum(lengths + 1, 0) - 1
    stream = torch.empty(n_tokens + n_sent, dtype=torch.int64, device=device)
    is_end = torch.zeros(n_tokens + n_sent, dtype=torch.bool, device=device)
    is_end[ends] = True
    stream[is_end] = 0
    stream[~is_end] = rows
    del rows
    stream = stream[stream >= 0].to(torch.int32)
    counts = np.concatenate([[n_sent], cnt[order].cpu().numpy()]).astype(np.uint32)
    gen_ids = order.cpu().numpy()
    words = [b"</s>"] + [b"w%d" % i for i in gen_ids.tolist()]
    return stream, counts, words, gen_ids
