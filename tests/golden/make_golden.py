"""Regenerate the golden fixtures from the reference itself.

Runs ``oracle/_ref/par_w2v_ref`` (the unmodified PAR_Word2Vec_cpu.cpp built by
``make -C oracle ref`` with the pinned-order SGEMM shim) at ``-threads 1`` on small seeded
corpora and stores, per case, under ``tests/golden/<case>/``:

    corpus.txt      the training text
    vocab.txt       the reference's vocabulary ("word count" in vocab order)
    win.npy/wout.npy  final W_in / W_out (float32, bit patterns of the reference run)
    exptable.npy    expTable[1001]
    output.txt      the reference's -output file (text format, "%f"; small cases only)
    meta.json       flags, vocab size, train_words, sha256 of the 1e8 unigram table and of W_in
                    as InitNet leaves it

Usage:  python tests/golden/make_golden.py   (needs the reference built; writes only here)
"""
from __future__ import annotations

import hashlib
import json
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from par_word2vec_b200 import synth  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref", "par_w2v_ref")


def _edge_corpus() -> bytes:
    long_word = b"x" * 130
    lines = [
        b"alpha beta gamma alpha beta\r\n",
        b"\tbeta  gamma\tdelta alpha " + long_word + b" beta\n",
        b"\n",
        b"   \n",
        b"gamma delta alpha beta gamma delta alpha beta " + long_word + b"\n",
    ]
    body = b"".join(lines * 40)
    body += b"rare1 rare2 alpha beta gamma delta epsilon alpha beta\n" * 3
    body += b"alpha beta gamma no_trailing_newline"
    return body


CASES = {
    # text8-like documents with topics, two epochs, subsampling, an empty line and a 2500-token line
    "text_small": dict(flags=dict(size=16, window=5, negative=5, sample="1e-3", iter=2, min_count=3,
                                  batch_size=24, alpha="0.025")),
    # random walks on a small DC-SBM graph: window 10, no subsampling (config 2 hyper-parameters)
    "graph_small": dict(flags=dict(size=32, window=10, negative=5, sample="0", iter=1, min_count=1,
                                   batch_size=24, alpha="0.025")),
    # tokenizer edge cases: CR, tabs, blank lines, 130-byte words, no trailing newline, tiny batches
    "edge": dict(flags=dict(size=8, window=3, negative=2, sample="1e-2", iter=3, min_count=2,
                            batch_size=4, alpha="0.05")),
    # text8-shaped hyper-parameters (d=100, w=5, n=5, sample 1e-4, batch 24)
    "d100": dict(flags=dict(size=100, window=5, negative=5, sample="1e-4", iter=1, min_count=5,
                            batch_size=24, alpha="0.025"), keep_output=False),
}


def corpus_bytes(case: str) -> bytes:
    tmp = tempfile.mkdtemp()
    try:
        path = os.path.join(tmp, "c.txt")
        if case == "text_small":
            toks, lens = synth.topic_zipf(200, 3000, 16, doc_len=100, seed=11)
            synth.write_text(path, toks, lens)
            with open(path, "ab") as f:
                f.write(b"\n" + b" ".join(b"w%d" % (i % 50) for i in range(2500)) + b"\n")
        elif case == "graph_small":
            toks, lens, _ = synth.dcsbm_walks(200, 5, 1500, walks_per_node=4, walk_len=20, seed=12)
            synth.write_text(path, toks, lens, prefix="n")
        elif case == "edge":
            with open(path, "wb") as f:
                f.write(_edge_corpus())
        elif case == "d100":
            toks, lens = synth.topic_zipf(300, 2000, 16, doc_len=200, seed=13)
            synth.write_text(path, toks, lens)
        with open(path, "rb") as f:
            return f.read()
    finally:
        shutil.rmtree(tmp)


def run_reference(corpus_path: str, flags: dict, workdir: str, threads: int = 1, dump_table: bool = True,
                  binary: str = REF) -> str:
    prefix = os.path.join(workdir, "r")
    args = [binary, "-train", corpus_path, "-output", os.path.join(workdir, "out.txt"), "-debug", "0",
            "-threads", str(threads), "-size", str(flags["size"]), "-window", str(flags["window"]),
            "-negative", str(flags["negative"]), "-sample", str(flags["sample"]), "-iter", str(flags["iter"]),
            "-min-count", str(flags["min_count"]), "-batch-size", str(flags["batch_size"]),
            "-alpha", str(flags["alpha"]), "-binary", "0", "-dump", prefix, "-dump-table", "1" if dump_table else "0"]
    subprocess.run(args, check=True, cwd=workdir, stdout=subprocess.DEVNULL)
    return prefix


def main() -> int:
    if not os.path.exists(REF):
        print("build the reference first: make -C oracle ref", file=sys.stderr)
        return 1
    for case, spec in CASES.items():
        out = os.path.join(HERE, case)
        os.makedirs(out, exist_ok=True)
        data = corpus_bytes(case)
        with open(os.path.join(out, "corpus.txt"), "wb") as f:
            f.write(data)
        work = tempfile.mkdtemp()
        try:
            prefix = run_reference(os.path.join(out, "corpus.txt"), spec["flags"], work)
            V, d, tw, fsz = map(int, open(prefix + ".meta").read().split())
            shutil.copy(prefix + ".vocab", os.path.join(out, "vocab.txt"))
            if spec.get("keep_output", True):
                shutil.copy(os.path.join(work, "out.txt"), os.path.join(out, "output.txt"))
            np.save(os.path.join(out, "win.npy"), np.fromfile(prefix + ".win", np.float32).reshape(V, d))
            np.save(os.path.join(out, "wout.npy"), np.fromfile(prefix + ".wout", np.float32).reshape(V, d))
            np.save(os.path.join(out, "exptable.npy"), np.fromfile(prefix + ".exptable", np.float32))
            table_sha = hashlib.sha256(open(prefix + ".table", "rb").read()).hexdigest()
            win0_sha = hashlib.sha256(open(prefix + ".win0", "rb").read()).hexdigest()
            meta = dict(flags=spec["flags"], vocab_size=V, size=d, train_words=tw, file_size=fsz,
                        table_sha256=table_sha, win0_sha256=win0_sha,
                        generator="tests/golden/make_golden.py", reference="PAR_Word2Vec_cpu.cpp -threads 1")
            with open(os.path.join(out, "meta.json"), "w") as f:
                json.dump(meta, f, indent=1, sort_keys=True)
            print(case, "V", V, "train_words", tw)
        finally:
            shutil.rmtree(work)
    return 0


if __name__ == "__main__":
    sys.exit(main())
