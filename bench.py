"""Words/sec of PAR-Word2Vec SGNS training on B200 (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload 1b|text8|graph] [--mode batched_bf16|batched|plain]

Workloads (synthetic stand-ins for the reference's public datasets, generated from a seed):
  1b     (default) 800M tokens, ~555k word types after min-count 5, topic-mixture Zipf(1.0) with
         256 topics, lognormal sentence lengths (mean 25, sigma 1, 1..1000); d=300, window 5,
         negative 5 shared per repulsion batch, sample 1e-4, batch 24, alpha 0.025, 1 iteration
         per step.  Generated on the device.  Default mode batched BF16.
  text8  17,000 documents of 1,000 tokens over 71,290 types, 64 topics; d=100, window 5,
         negative 5, sample 1e-4.  Default mode plain FP32 (the reference CPU program's own case).
  graph  uniform random walks (10 per node, length 80) over a DC-SBM graph of 10,312 nodes and
         39 communities; d=128, window 10, negative 5, no subsampling.  Default mode plain FP32.

A step is one training epoch over the whole corpus through the library's C ABI
(``parw2v_train``).  ``value`` times K steps with the corpus already on the device; ``e2e`` times
K steps of the user-facing sequence set_corpus (pinned host -> device) + train + get_weights
(W_in device -> pinned host).  For the 1b workload the corpus (3.3 GB) and the weights exceed the
126 MB L2, so no flush is needed between steps; the text8 and graph tables fit in L2 (their
roofline is the measured L2 read bandwidth) and the L2 is flushed before every step.  Several GPUs
run independent replicas (the training loop does not shard: every window updates the two shared
tables); ``value`` is the words of all replicas over the slowest replica's time.

The reference (PAR_Word2Vec_cpu.cpp built from its source into oracle/_ref by oracle/Makefile)
is timed on the host cores: on a 100M-token corpus of the same generator for the 1b workload
(with its corpus-load phase timed on its own) and on the whole corpus for text8 and graph; the
same run gives ``loss_vs_reference``.  ``--impl reference`` times it alone, on a bounded sample.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "words/sec on 1 B200: batched BF16 vs plain FP32 at equal planted-cluster recall"
WORKLOADS = {
    "1b": dict(hyper=dict(size=300, window=5, negative=5, batch_size=24, iter=1, alpha=0.025, sample=1e-4),
               mode="batched_bf16", n_types=555_000, n_topics=256, tokens=800_000_000,
               describe="1B-word-shaped corpus: 800M tokens, ~555k types after min-count 5, topic-mixture Zipf(1.0), "
                        "256 planted topics, lognormal sentences (mean 25, sigma 1, 1..1000)"),
    "text8": dict(hyper=dict(size=100, window=5, negative=5, batch_size=24, iter=1, alpha=0.025, sample=1e-4),
                  mode="plain", n_types=71_290, n_topics=64,
                  describe="text8-shaped corpus: 17,000 documents x 1,000 tokens over 71,290 types, 64 planted topics"),
    "graph": dict(hyper=dict(size=128, window=10, negative=5, batch_size=24, iter=1, alpha=0.025, sample=0.0),
                  mode="plain", n_nodes=10_312, n_comm=39,
                  describe="DC-SBM random walks: 10,312 nodes, 39 communities, ~334k edges, 10 walks x 80 per node"),
}
MIN_COUNT = 5
REF_SAMPLE_1B = 100_000_000   # tokens of the 1b generator the reference trains on in our arm
REF_ARM_SAMPLE = 20_000_000   # tokens per step of the reference arm (--impl reference)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="1b")
    ap.add_argument("--mode", default=None, choices=["plain", "batched", "batched_bf16"],
                    help="training mode timed (default: batched_bf16 for 1b, plain for text8 and graph)")
    ap.add_argument("--tokens", type=int, default=None, help="1b workload: corpus tokens (without </s>)")
    ap.add_argument("--no-compare", action="store_true", help="skip the other modes and the quality scores")
    ap.add_argument("--no-cpu-baseline", action="store_true", help="skip the reference CPU leg")
    ap.add_argument("--staging", default="auto", choices=["auto", "bulk", "cpasync"],
                    help="repulsion staging copies (parw2v_config.staging); the result does not depend on it")
    ap.add_argument("--attraction", default="default", choices=["default", "sequential", "pipelined"],
                    help="attraction form (parw2v_config.attraction); pipelined = sequential up to rounding")
    ap.add_argument("--autotune", type=int, default=0, help="parw2v_config.autotune")
    ap.add_argument("--variant", default="auto", choices=["auto", "stream", "window"],
                    help="BATCHED kernel organisation (parw2v_config.variant); the result does not depend on it")
    ap.add_argument("--min-rounds", type=int, default=0,
                    help="parw2v_config.min_rounds (0: the library's cap on sentences in flight; -1: no cap, "
                         "as the 800M-token corpus runs uncapped under the default)")
    a = ap.parse_args()
    a.mode = a.mode or WORKLOADS[a.workload]["mode"]
    return a


TRAFFIC_PROFILES = {"batched_bf16": "k_stream_train_bf16_10M_tokens.md", "batched": "k_stream_train_fp32_10M_tokens.md",
                    "plain": "k_plain_train_fp32_10M_tokens.md"}


def measured_traffic_per_kept_position(mode: str):
    """DRAM bytes per kept position of the training kernel, from the committed ncu summary of a
    10M-token capture of the same kernel (the 800M-token launch is too large to capture)."""
    import re
    name = TRAFFIC_PROFILES.get(mode)
    path = os.path.join(ROOT, "profiles", name) if name else None
    if not path or not os.path.exists(path):
        return None, None
    m = re.search(r"traffic_bytes_per_kept_position:\s*([0-9.]+)", open(path).read())
    return (float(m.group(1)), "profiles/" + name) if m else (None, None)


def measured_peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    return 6650.0, "fallback 6.65 TB/s (no MEASURED_PEAKS.json)"


def measured_l2_read_gbs(torch, device) -> float:
    """L2 read bandwidth measured here: a sum over a 32 MB buffer that stays in the 126 MB L2."""
    x = torch.ones(8 << 20, dtype=torch.float32, device=device)
    for _ in range(5):
        x.sum()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    n = 200
    for _ in range(n):
        x.sum()
    e1.record()
    torch.cuda.synchronize()
    return x.numel() * 4 * n / (e0.elapsed_time(e1) / 1e3) / 1e9


class ClockSampler:
    """nvidia-smi clock / throttle-reason samples while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.gpu)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(n):
    if n <= 1 or "RANK" not in os.environ:
        return None, 0, 1
    import torch.distributed as dist
    import datetime
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return dist, dist.get_rank(), dist.get_world_size()


def combine_replicas(torch, dist, words: int, ms: float, device: str = "cpu"):
    """Independent replicas: words of all ranks over the slowest rank's time."""
    if not dist:
        return words, ms
    t = torch.tensor([float(words), ms], dtype=torch.float64, device=device)
    w = t[:1].clone()
    dist.all_reduce(w, op=dist.ReduceOp.SUM)
    m = t[1:].clone()
    dist.all_reduce(m, op=dist.ReduceOp.MAX)
    return int(w.item()), float(m.item())


def timed_region(torch, dist, fn, steps, flush=None):
    """Barrier + synchronize, CUDA events around `steps` calls, synchronize + barrier; max over ranks.
    With `flush`, the L2 is flushed before every step; the flushes are timed apart and subtracted."""
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    out, ms = [], 0.0
    if flush is None:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        t0 = time.perf_counter()
        out = [fn() for _ in range(steps)]
        e1.record()
        torch.cuda.synchronize()
        ms = max(e0.elapsed_time(e1), (time.perf_counter() - t0) * 1e3)  # the library calls are synchronous
    else:
        for _ in range(steps):
            flush()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            t0 = time.perf_counter()
            out.append(fn())
            e1.record()
            torch.cuda.synchronize()
            ms += max(e0.elapsed_time(e1), (time.perf_counter() - t0) * 1e3)
    if dist:
        _, ms = combine_replicas(torch, dist, 0, ms, device="cuda")
        dist.barrier()
    return ms, out


def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def ref_flags(hyper: dict) -> dict:
    return dict(size=hyper["size"], window=hyper["window"], negative=hyper["negative"], sample=repr(hyper["sample"]),
                iter=hyper["iter"], min_count=MIN_COUNT, batch_size=hyper["batch_size"], alpha=repr(hyper["alpha"]))


def static_config(args) -> dict:
    wl = WORKLOADS[args.workload]
    return {"workload": wl["describe"], "mode": args.mode, **wl["hyper"], "min_count": MIN_COUNT}


# ---------------------------------------------------------------- the reference arm (CPU)

def reference_arm(args):
    """The reference's own CPU implementation on the host cores, on a bounded sample per step."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle import pwo, ref_run
    if not os.path.exists(pwo.REF_FAST_BIN):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/par_w2v_ref_fast is not built "
                                                              "(make -C oracle ref needs the reference sources)"}))
        return 0
    wl = WORKLOADS[args.workload]
    threads = host_threads()
    with tempfile.TemporaryDirectory() as tmp:
        corpus, vocab_file, note = make_reference_corpus(args, tmp, REF_ARM_SAMPLE)
        for _ in range(args.warmup):
            ref_run.run(corpus, ref_flags(wl["hyper"]), threads, read_vocab=vocab_file)
        words, secs, load = 0, 0.0, 0.0
        for _ in range(args.steps):
            r = ref_run.run(corpus, ref_flags(wl["hyper"]), threads, read_vocab=vocab_file, time_load=True)
            words += r["train_words"] * wl["hyper"]["iter"]
            secs += r["elapsed"]
            load += r["load_s"]
    value = words / secs
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "words/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": secs * 1e3 / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded, generated on the host)", "config": static_config(args),
            "cpu_baseline": {"value": value, "unit": "words/s", "cores": threads, "kind": "reference",
                             "sample": note + "; words/sec = corpus words x iter / the reference's own Elapsed "
                                                 "(its corpus load + training)",
                             "train_only_value": words / max(secs - load, 1e-9),
                             "load_s_per_step": load / args.steps},
            "e2e": {"value": value, "unit": "words/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def make_reference_corpus(args, tmp: str, tokens_1b: int):
    """Text corpus + vocabulary file the reference trains on; returns (corpus, vocab_file, note)."""
    from par_word2vec_b200 import synth
    from oracle import ref_run
    wl = WORKLOADS[args.workload]
    corpus = os.path.join(tmp, "corpus.txt")
    if args.workload == "1b":
        import torch
        dev = "cuda" if torch.cuda.is_available() else "cpu"
        stream_d, counts, words, _ = synth.topic_zipf_stream_torch(tokens_1b, wl["n_types"], wl["n_topics"], seed=4,
                                                                   min_count=MIN_COUNT, device=dev)
        stream = stream_d.cpu().numpy()
        del stream_d
        synth.write_stream_text(corpus, stream, words)
        vocab_file = os.path.join(tmp, "corpus.vocab")
        ref_run.write_vocab(vocab_file, words, counts)
        return corpus, vocab_file, (f"{tokens_1b} tokens (+{int(counts[0])} </s>) of the same generator, "
                                    f"{len(counts) - 1} types, vocabulary given to the reference by -read-vocab")
    if args.workload == "text8":
        toks, lens = synth.topic_zipf(17000, wl["n_types"], wl["n_topics"], doc_len=1000, seed=1)
        synth.write_text(corpus, toks, lens)
        return corpus, None, "the whole text8-shaped corpus (17M tokens), vocabulary learned by the reference"
    toks, lens, _ = synth.dcsbm_walks(seed=2)
    synth.write_text(corpus, toks, lens)
    return corpus, None, "the whole walk corpus (8.25M tokens), vocabulary learned by the reference"


# ---------------------------------------------------------------- our arm

def load_workload(args, torch, dev, tmp):
    """(stream_host_int32, counts, words, labels, corpus_text_or_None) for the workload."""
    import par_word2vec_b200 as pw
    from par_word2vec_b200 import evaluate, synth
    wl = WORKLOADS[args.workload]
    if args.workload == "1b":
        tokens = args.tokens or wl["tokens"]
        stream_d, counts, words, gen_ids = synth.topic_zipf_stream_torch(tokens, wl["n_types"], wl["n_topics"], seed=4,
                                                                         min_count=MIN_COUNT, device=dev)
        stream_h = torch.empty(int(stream_d.numel()), dtype=torch.int32, pin_memory=True)
        stream_h.copy_(stream_d)
        del stream_d
        torch.cuda.empty_cache()
        labels = np.full(len(counts), -1, np.int64)
        labels[1:] = gen_ids % wl["n_topics"]
        return stream_h, counts, words, labels, None
    corpus = os.path.join(tmp, "corpus.txt")
    if args.workload == "text8":
        toks, lens = synth.topic_zipf(17000, wl["n_types"], wl["n_topics"], doc_len=1000, seed=1)
        synth.write_text(corpus, toks, lens)
    else:
        toks, lens, comm = synth.dcsbm_walks(seed=2)
        synth.write_text(corpus, toks, lens)
    vocab = pw.Vocab.learn(corpus, MIN_COUNT)
    stream = vocab.load_stream(corpus)
    words = vocab.words()
    counts = vocab.counts()
    if args.workload == "text8":
        labels = evaluate.labels_from_words(words, wl["n_topics"])
    else:
        labels = np.array([comm[int(w[1:])] if w.startswith(b"w") else -1 for w in words], np.int64)
    stream_h = torch.empty(len(stream), dtype=torch.int32, pin_memory=True)
    stream_h.numpy()[:] = stream
    return stream_h, counts, words, labels, corpus


def main():
    args = parse()
    if args.impl == "reference":
        return reference_arm(args)
    import torch
    import par_word2vec_b200 as pw
    from par_word2vec_b200 import evaluate

    dist, rank, world = dist_setup(args.gpus)
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = f"cuda:{local}"
    wl = WORKLOADS[args.workload]
    hyper = wl["hyper"]
    d = hyper["size"]
    tmp = tempfile.mkdtemp()
    stream_h, counts, words, labels, corpus_text = load_workload(args, torch, dev, tmp)
    stream_np = stream_h.numpy()
    n = len(stream_np)
    n_sent = int(counts[0])  # one "</s>" per sentence
    V = len(counts)
    mode = pw.MODE_NAMES[args.mode]
    bytes_per = 2 if mode == pw.MODE_BATCHED_BF16 else 4
    staging = {"auto": pw.STAGING_AUTO, "bulk": pw.STAGING_BULK, "cpasync": pw.STAGING_CPASYNC}[args.staging]
    l2_resident = args.workload != "1b"
    flush_buf = torch.empty(256 << 20, dtype=torch.uint8, device=dev) if l2_resident else None

    def flush():
        flush_buf.add_(1)  # a 256 MB write: evicts the 126 MB L2

    attraction = {"default": pw.ATTRACT_DEFAULT, "sequential": pw.ATTRACT_SEQUENTIAL,
                  "pipelined": pw.ATTRACT_PIPELINED}[args.attraction]

    def make(m, seed, min_rounds=None, stream=stream_np):
        variant = {"auto": pw.VARIANT_AUTO, "stream": pw.VARIANT_STREAM, "window": pw.VARIANT_WINDOW}[args.variant]
        t = pw.Trainer(mode=m, device=local, seed=seed, staging=staging, attraction=attraction, autotune=args.autotune,
                       variant=variant,
                       min_rounds=args.min_rounds if min_rounds is None else min_rounds, **hyper)
        t.set_vocab(counts)
        t.init_weights()
        t.set_corpus(stream)
        return t

    tr = make(mode, 1 + rank)
    for _ in range(args.warmup):
        tr.train()
    with ClockSampler(local) as clk:
        ms, stats = timed_region(torch, dist, tr.train, args.steps, flush if l2_resident else None)
    words_all = n * args.steps * world
    value = words_all / (ms / 1e3)

    # roofline of the dominant kernel (the training kernel), from its CUDA-event time per launch
    mean = lambda k: sum(s[k] for s in stats) / len(stats)  # noqa: E731
    kernel_ms, kept, negs, pairs = mean("kernel_ms"), mean("kept"), mean("negatives"), mean("pairs")
    alg_bytes = kept * (4 * bytes_per * d + 4) + negs * (2 * bytes_per * d + 4)
    pair_bytes = 2 * bytes_per * d * (2 * pairs + kept + negs)
    achieved = alg_bytes / (kernel_ms / 1e3) / 1e9
    if l2_resident:
        peak, peak_src, bound = measured_l2_read_gbs(torch, dev), "measured here: L2 read bandwidth (32 MB buffer)", "l2"
    else:
        (peak, peak_src), bound = measured_peak_hbm(), "hbm"
    tpp, tsrc = measured_traffic_per_kept_position(args.mode) if args.workload == "1b" else (None, None)
    roofline = {"bound": bound, "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": tpp * kept if tpp else None, "kernel": "training kernel", "peak_source": peak_src,
                "alg_bytes_per_launch": alg_bytes, "kernel_ms_per_launch": kernel_ms,
                "pack_ms_per_launch": mean("pack_ms"), "alg_bytes_per_kept_position": alg_bytes / max(kept, 1),
                "pair_bytes_per_kept_position": pair_bytes / max(kept, 1),
                "pair_bytes_note": "B_pair = 2 s d (2 pairs + kept + negatives): every pair's two rows read and "
                                   "written, an upper bound on row traffic at the reference's granularity",
                "traffic_note": (f"ncu dram__bytes_read+write per kept position of the same kernel ({tsrc}, a "
                                 f"10M-token capture) x kept positions of this launch" if tpp else
                                 "no ncu capture of this workload")}

    # ---- end to end through the C ABI with host buffers ----
    w_host = torch.empty((V, d), dtype=torch.float32, pin_memory=True).numpy()  # pinned, like the corpus

    def e2e_step():
        tr.set_corpus(stream_np)
        st = tr.train()
        tr._check(tr._lib.parw2v_get_weights(tr._h, w_host.ctypes.data, None))  # into the pinned buffer
        return st

    e2e_ms, _ = timed_region(torch, dist, e2e_step, args.steps, flush if l2_resident else None)
    e2e = {"value": words_all / (e2e_ms / 1e3), "unit": "words/s", "h2d_bytes_per_step": 4 * n,
           "d2h_bytes_per_step": 4 * V * d}
    tr.close()

    cfg = static_config(args)
    cfg.update({"corpus_tokens_with_eos": n, "sentences": n_sent, "vocab_size": V, "min_rounds": args.min_rounds,
                "staging": args.staging, "attraction": args.attraction, "autotune": args.autotune,
                "variant": args.variant,
                "replicas": world, "launch": {k: stats[0][k] for k in ("grid", "warps_per_cta", "variant", "lane_elems",
                                                                        "staging", "attraction", "repulsion")},
                "l2": ("flushed before every step (256 MB write, outside the timed events); the tables fit in L2"
                       if l2_resident else "no flush: corpus (4 B/token) and weights exceed the 126 MB L2")})
    line = {"metric": METRIC, "value": value, "unit": "words/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "bf16" if bytes_per == 2 else "f32",
            "data": "synthetic (seeded; " + ("generated on the device)" if not l2_resident else
                                             "generated on the host, read by the library's reference-identical "
                                             "front end)"),
            "config": cfg, "roofline": roofline, "e2e": e2e, "gpu_launches": int(args.steps * (1 + hyper["iter"] * 4)),
            "clocks": clk.summary(),
            "stats_per_step": {k: stats[0][k] for k in ("words", "kept", "sentences", "pairs", "batches", "negatives")}}

    if rank == 0 and not args.no_compare:
        # quality of each mode after ONE epoch from InitNet, on the same corpus and evaluation set
        queries = evaluate.top_queries(counts, labels, 10000)
        rare = evaluate.top_queries(counts, labels, 400_000)[200_000:] if args.workload == "1b" else None
        triples = evaluate.eval_triples(stream_np, counts, n_windows=4096, window=hyper["window"])

        def quality(m):
            t = make(m, 1)
            st = t.train()
            w_in, w_out = t.get_weights()
            t.close()
            q = {"words_per_s_one_epoch": n / (st["kernel_ms"] + st["pack_ms"]) * 1e3,
                 "loss": score_loss(pw, evaluate, counts, hyper, w_in, w_out, triples),
                 "recall_at_10": evaluate.recall_at_10(w_in, labels, queries, device=dev)}
            q["topic_margin"] = evaluate.topic_margin(w_in, labels, queries, device=dev)
            if rare is not None:
                q["topic_margin_rank_200k_400k"] = evaluate.topic_margin(w_in, labels, rare, device=dev)
            return q

        modes = ["batched_bf16", "plain", "batched"]
        line["quality_one_epoch"] = {m: quality(pw.MODE_NAMES[m]) for m in modes}
        q = line["quality_one_epoch"]
        line["speedup_vs_plain"] = value / q["plain"]["words_per_s_one_epoch"]
        line["quality_note"] = ("each mode trained one epoch from InitNet on this corpus in a fresh context; loss = "
                                "mean SGNS loss on 4,096 fixed windows; recall@10 over the 10,000 most frequent words; "
                                "topic_margin = cosine to the own planted topic's centroid minus the mean cosine to the "
                                "other centroids (continuous, where recall@10 saturates)"
                                + ("; topic_margin_rank_200k_400k over frequency ranks 200,000-400,000"
                                   if rare is not None else ""))
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line.update(reference_leg(args, pw, evaluate, hyper, dev, tmp, corpus_text, stream_np, counts, words, labels))
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def knob_kwargs(args, pw) -> dict:
    """The launch knobs of this run (result-neutral), as Trainer keyword arguments."""
    return dict(staging={"auto": pw.STAGING_AUTO, "bulk": pw.STAGING_BULK, "cpasync": pw.STAGING_CPASYNC}[args.staging],
                attraction={"default": pw.ATTRACT_DEFAULT, "sequential": pw.ATTRACT_SEQUENTIAL,
                            "pipelined": pw.ATTRACT_PIPELINED}[args.attraction],
                variant={"auto": pw.VARIANT_AUTO, "stream": pw.VARIANT_STREAM, "window": pw.VARIANT_WINDOW}[args.variant],
                autotune=args.autotune)


def score_loss(pw, evaluate, counts, hyper, w_in, w_out, triples) -> float:
    with pw.Trainer(size=hyper["size"], mode=pw.MODE_PLAIN) as t:
        t.set_vocab(counts)
        t.set_weights(w_in, w_out)
        return evaluate.sgns_loss(t, triples)


def reference_leg(args, pw, evaluate, hyper, dev, tmp, corpus_text, stream_np, counts, words, labels) -> dict:
    """cpu_baseline and loss_vs_reference: the reference on the host cores and our timed mode on the
    same corpus, one run each, scored on the same evaluation windows."""
    from oracle import pwo, ref_run
    if not os.path.exists(pwo.REF_FAST_BIN):
        return {"cpu_baseline": None, "cpu_baseline_note": "oracle/_ref not built"}
    threads = host_threads()
    if args.workload == "1b":
        corpus, vocab_file, note = make_reference_corpus(args, tmp, REF_SAMPLE_1B)
        # the same generator's 100M-token corpus in our vocabulary order, for our run beside it
        import torch
        from par_word2vec_b200 import synth
        wl = WORKLOADS["1b"]
        sd, c2, w2, g2 = synth.topic_zipf_stream_torch(REF_SAMPLE_1B, wl["n_types"], wl["n_topics"], seed=4,
                                                       min_count=MIN_COUNT, device=dev)
        s2 = sd.cpu().numpy()
        del sd
        torch.cuda.empty_cache()
        l2 = np.full(len(c2), -1, np.int64)
        l2[1:] = g2 % wl["n_topics"]
        # the library's default concurrency for this corpus (about 490 sentences in flight): at a
        # fixed number in flight the loss moves with corpus size, so the bench's own concurrency
        # (2,368) is compared on the 800M-token corpus itself, in tests/test_headline_gpu.py
        ours_min_rounds = 0
    else:
        corpus, vocab_file, note = corpus_text, None, f"the whole {args.workload} corpus, vocabulary learned by the reference"
        s2, c2, w2, l2 = stream_np, counts, words, labels
        ours_min_rounds = args.min_rounds
    r = ref_run.run(corpus, ref_flags(hyper), threads, read_vocab=vocab_file, time_load=True)
    ref_win, ref_wout = ref_run.rows_in_order(r, w2)
    triples = evaluate.eval_triples(s2, c2, n_windows=4096, window=hyper["window"])
    queries = evaluate.top_queries(c2, l2, 10000)
    mode = pw.MODE_NAMES[args.mode]
    with pw.Trainer(mode=mode, seed=1, min_rounds=ours_min_rounds, **knob_kwargs(args, pw), **hyper) as t:
        t.set_vocab(c2)
        t.init_weights()
        t.set_corpus(s2)
        t.train()
        w_in, w_out = t.get_weights()
    ours_loss = score_loss(pw, evaluate, c2, hyper, w_in, w_out, triples)
    ref_loss = score_loss(pw, evaluate, c2, hyper, ref_win, ref_wout, triples)
    words_ref = r["train_words"] * hyper["iter"]
    extra = {}
    if args.workload == "graph" and os.path.exists(ref_run.GPU_GRAPH_BIN):
        # the reference's own GPU program on the same walks: the GPU-vs-GPU comparison
        g = ref_run.run_gpu_graph(corpus, ref_flags(hyper), int(c2[0]))
        pos = {w: i for i, w in enumerate(g["words"])}
        g_win = g["win"][np.array([pos[w] for w in w2])]
        extra["gpu_reference"] = {
            "value": words_ref / g["elapsed"], "unit": "words/s", "device_s": g["elapsed"],
            "recall_at_10": evaluate.recall_at_10(g_win, l2, queries, device=dev),
            "note": "PAR_Word2Vec_gpu_graph.cu built for sm_100a (oracle/Makefile ref-gpu), default -gamma 32, "
                    "its own CUDA-event time of its training kernel; it draws negatives uniformly and keeps "
                    "alpha fixed within an epoch, so its loss is not comparable (it saves W_in only)"}
    return {**extra,
        "cpu_baseline": {"value": words_ref / r["elapsed"], "unit": "words/s", "cores": threads, "kind": "reference",
                         "sample": note + "; words/sec = corpus words x iter / the reference's own Elapsed (its "
                                          "per-thread corpus load + training)",
                         "train_only_value": words_ref / max(r["elapsed"] - r["load_s"], 1e-9),
                         "load_s": r["load_s"], "elapsed_s": r["elapsed"]},
        "loss_vs_reference": {"ours": ours_loss, "reference": ref_loss, "rel": ours_loss / ref_loss - 1.0,
                              "ours_recall_at_10": evaluate.recall_at_10(w_in, l2, queries, device=dev),
                              "reference_recall_at_10": evaluate.recall_at_10(ref_win, l2, queries, device=dev),
                              "ours_topic_margin": evaluate.topic_margin(w_in, l2, queries, device=dev),
                              "reference_topic_margin": evaluate.topic_margin(ref_win, l2, queries, device=dev),
                              "note": f"{args.mode} (min_rounds {ours_min_rounds}) and one reference run at {threads} "
                                      f"threads on the corpus above; bar 1% (the reference's own runs spread ~0.8%)"},
    }


if __name__ == "__main__":
    sys.exit(main())
