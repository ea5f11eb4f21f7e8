"""TEST INFRASTRUCTURE ONLY: runs the reference binaries built by oracle/Makefile -- the CPU
program PAR_Word2Vec_cpu.cpp (oracle/_ref/par_w2v_ref_fast, through its dumping driver) and the GPU
graph program PAR_Word2Vec_gpu_graph.cu (oracle/_ref/par_w2v_gpu_graph) -- and reads back their
outputs.

Only tests/ and bench.py's CPU-baseline / reference legs use this module, as the checker and the
timed CPU baseline; nothing in the library imports it.
"""
from __future__ import annotations

import os
import re
import subprocess
import tempfile

import numpy as np

from oracle import pwo


def write_vocab(path: str, words: list[bytes], counts: np.ndarray) -> None:
    """A vocabulary file in the reference's SaveVocab format ("word count" per line,
    PAR_Word2Vec_cpu.cpp:294-299), "</s>" first, for its -read-vocab (ReadVocab, :301-335)."""
    with open(path, "wb") as f:
        f.write(b"".join(w + b" %d\n" % int(c) for w, c in zip(words, counts.tolist())))


def run(corpus: str, flags: dict, threads: int, read_vocab: str | None = None, time_load: bool = False,
        binary: str | None = None) -> dict:
    """One run of the reference on `corpus` with its command-line `flags` (names without the dash).

    Returns W_in / W_out in the reference's vocabulary order, its words, its own ``Elapsed``
    seconds (corpus load + training, PAR_Word2Vec_cpu.cpp:395-706) and, with time_load, the
    seconds of the load phase alone (timed by the driver with the reference's own loadStream)."""
    exe = binary or pwo.REF_FAST_BIN
    if not os.path.exists(exe):
        raise FileNotFoundError(f"{exe} is not built (make -C oracle ref)")
    with tempfile.TemporaryDirectory() as tmp:
        args = [exe, "-train", corpus, "-output", os.path.join(tmp, "o.bin"), "-binary", "1", "-debug", "0",
                "-threads", str(threads), "-dump", os.path.join(tmp, "r")]
        if read_vocab:
            args += ["-read-vocab", read_vocab]
        if time_load:
            args += ["-time-load", "1"]
        for k, v in flags.items():
            args += ["-" + k.replace("_", "-"), str(v)]
        env = dict(os.environ, OMP_PROC_BIND="close")
        subprocess.run(args, check=True, cwd=tmp, stdout=subprocess.DEVNULL, env=env)
        V, d, train_words, _ = map(int, open(os.path.join(tmp, "r.meta")).read().split())
        words = [ln.rsplit(b" ", 1)[0] for ln in open(os.path.join(tmp, "r.vocab"), "rb").read().splitlines()]
        out = dict(V=V, d=d, train_words=train_words, words=words,
                   win=np.fromfile(os.path.join(tmp, "r.win"), np.float32).reshape(V, d),
                   wout=np.fromfile(os.path.join(tmp, "r.wout"), np.float32).reshape(V, d))
        out["elapsed"] = float(re.search(rb"Elapsed\s+([0-9.]+)",
                                         open(os.path.join(tmp, "PAR_Word2Vec_cpu_time"), "rb").read()).group(1))
        if time_load:
            out["load_s"] = float(open(os.path.join(tmp, "r.load")).read())
    return out


def rows_in_order(ref: dict, words: list[bytes]):
    """The reference's W_in / W_out rows permuted into the row order of `words` (same word set)."""
    pos = {w: i for i, w in enumerate(ref["words"])}
    idx = np.array([pos[w] for w in words], dtype=np.int64)
    return ref["win"][idx], ref["wout"][idx]


GPU_GRAPH_BIN = os.path.join(os.path.dirname(pwo.REF_FAST_BIN), "par_w2v_gpu_graph")


def read_binary_vectors(path: str):
    """A saveModel file written with -binary 1 (PAR_Word2Vec_gpu_graph.cu saveModel): a "V d" header
    line, then per word its string, a space, d float32 values and a newline."""
    data = open(path, "rb").read()
    nl = data.index(b"\n")
    V, d = map(int, data[:nl].split())
    pos, words = nl + 1, []
    W = np.empty((V, d), np.float32)
    for i in range(V):
        sp = data.index(b" ", pos)
        words.append(data[pos:sp])
        W[i] = np.frombuffer(data, np.float32, d, sp + 1)
        pos = sp + 1 + 4 * d + 1
    return words, W


def run_gpu_graph(corpus: str, flags: dict, n_sentences: int) -> dict:
    """One run of the reference's GPU graph program (hidden size 128 only: its kernel reads four
    32-wide slices of each row) on the first visible device, in this process's environment.
    Returns its device time ``elapsed`` (its own CUDA-event Elapsed,
    PAR_Word2Vec_gpu_graph.cu:869-957), W_in and the words in its row order."""
    if not os.path.exists(GPU_GRAPH_BIN):
        raise FileNotFoundError(f"{GPU_GRAPH_BIN} is not built (make -C oracle ref-gpu)")
    with tempfile.TemporaryDirectory() as tmp:
        out = os.path.join(tmp, "o.bin")
        # -max-num-sen sizes its host array of sentence offsets: at least the corpus's lines
        args = [GPU_GRAPH_BIN, "-train", corpus, "-output", out, "-binary", "1", "-debug", "0",
                "-max-num-sen", str(n_sentences + 16)]
        for k, v in flags.items():
            args += ["-" + k.replace("_", "-"), str(v)]
        subprocess.run(args, check=True, cwd=tmp, stdout=subprocess.DEVNULL)
        elapsed = float(re.search(rb"Elapsed\s+([0-9.]+)",
                                  open(os.path.join(tmp, "PAR_Word2Vec_gpu_time"), "rb").read()).group(1))
        words, W = read_binary_vectors(out)
    return dict(elapsed=elapsed, words=words, win=W)
