"""Words/sec of PAR-Word2Vec SGNS training on B200 (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--mode batched_bf16]

Workload (synthetic stand-in for the 1B-word benchmark, generated on the device from a seed):
800M tokens, ~555k word types after min-count 5, topic-mixture Zipf(1.0) with 256 topics,
lognormal sentence lengths (mean 25, sigma 1, 1..1000); d=300, window 5, negative 5 shared per
repulsion batch, sample 1e-4, batch 24, alpha 0.025, 1 iteration per step.

A step is one training epoch over the whole corpus through the library's C ABI
(``parw2v_train``).  ``value`` times K steps with the corpus already on the device; ``e2e``
times K steps of the user-facing sequence set_corpus (pinned host -> device) + train +
get_weights (W_in device -> pinned host).  The corpus (3.2 GB) and weights exceed the 126 MB L2, so no
L2 flush is inserted between steps.  Several GPUs run independent replicas (the training loop
does not shard: every window updates the two shared tables); ``value`` is the words of all
replicas over the slowest replica's time.

``--impl reference`` times the reference's own CPU implementation (PAR_Word2Vec_cpu.cpp built
from its source into oracle/_ref) on a bounded sample of the same corpus with all host threads.
"""
from __future__ import annotations

import argparse
import json
import os
import re
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
HYPER = dict(size=300, window=5, negative=5, batch_size=24, iter=1, alpha=0.025, sample=1e-4)
N_TYPES, N_TOPICS, MIN_COUNT = 555_000, 256, 5


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--mode", default="batched_bf16", choices=["plain", "batched", "batched_bf16"])
    ap.add_argument("--tokens", type=int, default=800_000_000, help="corpus tokens (without </s>)")
    ap.add_argument("--no-compare", action="store_true", help="skip the plain FP32 comparison and recall")
    ap.add_argument("--cpu-sample", type=int, default=6_000_000, help="tokens in the CPU-baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--min-rounds", type=int, default=0,
                    help="parw2v_config.min_rounds (0: the library's cap on sentences in flight; -1: no cap, "
                         "as the 800M-token corpus runs uncapped under the default)")
    return ap.parse_args()


def measured_traffic_per_kept_position(mode: str):
    """DRAM bytes per kept position of the training kernel, from the committed ncu summary."""
    name = {"batched_bf16": "k_stream_train_bf16_10M_tokens.md"}.get(mode)
    if not name:
        return None, None
    path = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(path):
        return None, None
    m = re.search(r"traffic_bytes_per_kept_position:\s*([0-9.]+)", open(path).read())
    return (float(m.group(1)), "profiles/" + name) if m else (None, None)


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    return 6650.0, "fallback 6.65 TB/s"


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


def timed_region(torch, dist, fn, steps):
    """Barrier + synchronize, CUDA events around `steps` calls, synchronize + barrier; max over ranks."""
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    t0 = time.perf_counter()
    out = [fn() for _ in range(steps)]
    e1.record()
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    ms = max(e0.elapsed_time(e1), wall * 1e3)  # the library calls are synchronous; both agree
    if dist:
        _, ms = combine_replicas(torch, dist, 0, ms, device="cuda")
        dist.barrier()
    return ms, out


def write_sample_text(path: str, stream: np.ndarray, words: list[bytes], n_tokens: int) -> int:
    """The first n_tokens of the stream (whole sentences) as reference-readable text."""
    zeros = np.flatnonzero(stream[: n_tokens + 2000] == 0)
    end = int(zeros[np.searchsorted(zeros, n_tokens)]) + 1 if len(zeros) else n_tokens
    part = stream[:end]
    names = np.array(words, dtype=object)
    with open(path, "wb") as f:
        cuts = np.flatnonzero(part == 0)
        start = 0
        buf = []
        for c in cuts.tolist():
            buf.append(b" ".join(names[part[start:c]].tolist()))
            start = c + 1
            if len(buf) >= 8192:
                f.write(b"\n".join(buf) + b"\n")
                buf = []
        if buf:
            f.write(b"\n".join(buf) + b"\n")
    return end


def run_reference_cpu(sample_path: str, threads: int):
    """The reference binary on the sample; returns (words/sec by its Elapsed timer, elapsed, train_words)."""
    from oracle import pwo
    exe = pwo.REF_FAST_BIN
    if not os.path.exists(exe):
        return None
    with tempfile.TemporaryDirectory() as tmp:
        args = [exe, "-train", sample_path, "-output", os.path.join(tmp, "o.bin"), "-binary", "1", "-debug", "0",
                "-threads", str(threads), "-dump", os.path.join(tmp, "r"), "-size", str(HYPER["size"]),
                "-window", str(HYPER["window"]), "-negative", str(HYPER["negative"]),
                "-sample", str(HYPER["sample"]), "-iter", str(HYPER["iter"]), "-min-count", str(MIN_COUNT),
                "-batch-size", str(HYPER["batch_size"]), "-alpha", str(HYPER["alpha"])]
        env = dict(os.environ, OMP_PROC_BIND="close")
        subprocess.run(args, check=True, cwd=tmp, stdout=subprocess.DEVNULL, env=env)
        elapsed = float(re.search(rb"Elapsed\s+([0-9.]+)", open(os.path.join(tmp, "PAR_Word2Vec_cpu_time"), "rb").read()).group(1))
        V, d, tw, _ = map(int, open(os.path.join(tmp, "r.meta")).read().split())
    return tw * HYPER["iter"] / max(elapsed, 1e-3), elapsed, tw


def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from par_word2vec_b200 import synth
    toks, lens = synth.topic_zipf(args.cpu_sample, N_TYPES, N_TOPICS, doc_len=None, lognormal_mean=25.0, seed=4)
    threads = host_threads()
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "sample.txt")
        synth.write_text(path, toks, lens)
        for _ in range(args.warmup):
            run_reference_cpu(path, threads)
        words, secs = 0, 0.0
        for _ in range(args.steps):
            r = run_reference_cpu(path, threads)
            words += r[2]
            secs += r[1]
    value = words / secs
    sample = (f"{args.cpu_sample} tokens of the same generator (lognormal sentences, 256 topics), "
              f"reference vocabulary after min-count 5; words/sec by the reference's own Elapsed timer "
              f"(corpus load + training)")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "words/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": secs * 1e3 / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded, generated on the host)",
            "config": {"workload": "1B-word-shaped corpus, bounded CPU sample", **HYPER, "min_count": MIN_COUNT},
            "cpu_baseline": {"value": value, "unit": "words/s", "cores": threads, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": value, "unit": "words/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return reference_arm(args)
    import torch
    import par_word2vec_b200 as pw
    from par_word2vec_b200 import evaluate, synth

    dist, rank, world = dist_setup(args.gpus)
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = f"cuda:{local}"

    # ---- workload (device generation, host copy in pinned memory) ----
    stream_d, counts, words, gen_ids = synth.topic_zipf_stream_torch(args.tokens, N_TYPES, N_TOPICS,
                                                                       seed=4, min_count=MIN_COUNT, device=dev)
    n = int(stream_d.numel())
    n_sent = int(counts[0])  # one "</s>" per sentence
    stream_h = torch.empty(n, dtype=torch.int32, pin_memory=True)
    stream_h.copy_(stream_d)
    del stream_d
    torch.cuda.empty_cache()
    stream_np = stream_h.numpy()
    V = len(counts)
    mode = pw.MODE_NAMES[args.mode]
    bytes_per = 2 if mode == pw.MODE_BATCHED_BF16 else 4
    d = HYPER["size"]

    def make(m, seed):
        t = pw.Trainer(mode=m, device=local, seed=seed, min_rounds=args.min_rounds, **HYPER)
        t.set_vocab(counts)
        t.init_weights()
        t.set_corpus(stream_np)
        return t

    tr = make(mode, 1 + rank)
    for _ in range(args.warmup):
        tr.train()
    with ClockSampler(local) as clk:
        ms, stats = timed_region(torch, dist, tr.train, args.steps)
    words_all = n * args.steps * world
    value = words_all / (ms / 1e3)

    # roofline of the dominant kernel (the training kernel), from its CUDA-event time per launch
    kernel_ms = sum(s["kernel_ms"] for s in stats) / len(stats)
    kept = sum(s["kept"] for s in stats) / len(stats)
    negs = sum(s["negatives"] for s in stats) / len(stats)
    alg_bytes = kept * (4 * bytes_per * d + 4) + negs * (2 * bytes_per * d + 4)
    achieved = alg_bytes / (kernel_ms / 1e3) / 1e9
    peak, peak_src = measured_peaks()
    tpp, tsrc = measured_traffic_per_kept_position(args.mode)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": tpp * kept if tpp else None,
                "traffic_source": (f"ncu dram__bytes_read+write per kept position ({tsrc}, 10M-token capture) "
                                   f"x kept positions per launch") if tpp else None,
                "kernel": "training kernel", "peak_source": peak_src,
                "alg_bytes_per_launch": alg_bytes, "kernel_ms_per_launch": kernel_ms,
                "pack_ms_per_launch": sum(s["pack_ms"] for s in stats) / len(stats),
                "alg_bytes_per_kept_position": alg_bytes / max(kept, 1)}

    # ---- end to end through the C ABI with host buffers ----
    w_host = torch.empty((V, d), dtype=torch.float32, pin_memory=True).numpy()  # pinned, like the corpus

    def e2e_step():
        tr.set_corpus(stream_np)
        st = tr.train()
        tr._check(tr._lib.parw2v_get_weights(tr._h, w_host.ctypes.data, None))  # into the pinned buffer
        return st

    e2e_ms, _ = timed_region(torch, dist, e2e_step, args.steps)
    e2e = {"value": words_all / (e2e_ms / 1e3), "unit": "words/s", "h2d_bytes_per_step": 4 * n,
           "d2h_bytes_per_step": 4 * V * d}
    w_in_final = w_host.copy()
    tr.close()

    line = {"metric": METRIC, "value": value, "unit": "words/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "bf16" if bytes_per == 2 else "f32",
            "data": "synthetic (seeded topic-mixture Zipf corpus generated on the device)",
            "config": {"workload": f"1B-word-shaped corpus: {n - n_sent} tokens (of {args.tokens} generated, "
                                   f"words under min-count {MIN_COUNT} dropped) + {n_sent} </s>, "
                                   f"{V - 1} word types, 256 planted topics",
                       "mode": args.mode, **HYPER, "min_count": MIN_COUNT, "min_rounds": args.min_rounds,
                       "corpus_tokens_with_eos": n,
                       "vocab_size": V, "replicas": world,
                       "l2": "no flush: corpus (4 B/token) and weights exceed the 126 MB L2"},
            "roofline": roofline, "e2e": e2e, "gpu_launches": int(args.steps * (1 + HYPER["iter"] * 4)),
            "clocks": clk.summary(),
            "stats_per_step": {k: stats[0][k] for k in ("words", "kept", "sentences", "pairs", "batches", "negatives")}}

    if rank == 0 and not args.no_compare:
        labels = np.full(V, -1, np.int64)
        labels[1:] = gen_ids % N_TOPICS
        queries = evaluate.top_queries(counts, labels, 10000)
        line["recall_at_10"] = evaluate.recall_at_10(w_in_final, labels, queries, device=dev)
        if mode != pw.MODE_PLAIN:
            tp = make(pw.MODE_PLAIN, 1)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            st = tp.train()
            p_ms = (time.perf_counter() - t0) * 1e3
            w_plain = tp.get_weights("in")
            tp.close()
            line["plain_fp32"] = {"value": n / (p_ms / 1e3), "unit": "words/s", "kernel_ms": st["kernel_ms"],
                                  "recall_at_10": evaluate.recall_at_10(w_plain, labels, queries, device=dev),
                                  "steps": 1, "note": "first epoch from InitNet, same corpus"}
            line["speedup_vs_plain"] = value / line["plain_fp32"]["value"]
        if mode == pw.MODE_BATCHED_BF16:
            # the batched FP32 configuration on the same corpus (FP32 tables, same kernels otherwise)
            tf = make(pw.MODE_BATCHED, 1)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            st = tf.train()
            f_ms = (time.perf_counter() - t0) * 1e3
            w_f32 = tf.get_weights("in")
            tf.close()
            line["batched_fp32"] = {"value": n / (f_ms / 1e3), "unit": "words/s", "kernel_ms": st["kernel_ms"],
                                    "recall_at_10": evaluate.recall_at_10(w_f32, labels, queries, device=dev),
                                    "steps": 1, "note": "first epoch from InitNet, same corpus"}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = host_threads()
        with tempfile.TemporaryDirectory() as tmp:
            path = os.path.join(tmp, "sample.txt")
            write_sample_text(path, stream_np, words, args.cpu_sample)
            r = run_reference_cpu(path, threads)
        if r:
            line["cpu_baseline"] = {"value": r[0], "unit": "words/s", "cores": threads, "kind": "reference",
                                    "sample": f"first {r[2]} corpus tokens (whole sentences) as text; reference "
                                              f"vocabulary of the sample; its own Elapsed timer (load + train)"}
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
