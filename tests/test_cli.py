"""The parw2v command line as a drop-in for the reference binaries."""
import os
import subprocess
import tempfile

import pytest

from tests.conftest import ROOT

CLI = os.path.join(ROOT, "par_word2vec_b200", "bin", "parw2v")


def run_cli(args, cwd):
    return subprocess.run([CLI] + args, cwd=cwd, capture_output=True, text=True)


def flag_args(g):
    f = g.flags
    return ["-size", str(f["size"]), "-window", str(f["window"]), "-negative", str(f["negative"]),
            "-sample", str(f["sample"]), "-iter", str(f["iter"]), "-min-count", str(f["min_count"]),
            "-batch-size", str(f["batch_size"]), "-alpha", str(f["alpha"]), "-threads", "1", "-debug", "0"]


def test_usage_and_missing_train():
    with tempfile.TemporaryDirectory() as t:
        r = run_cli([], t)
        assert r.returncode == 0 and "-train" in r.stdout
        r = run_cli(["-output", "x"], t)
        assert r.returncode != 0


def test_save_vocab_only_matches_reference(golden):
    """Without -output the reference stops after the vocabulary (PAR_Word2Vec_cpu.cpp:384-385)."""
    with tempfile.TemporaryDirectory() as t:
        v = os.path.join(t, "vocab.txt")
        r = run_cli(["-train", golden.corpus_path, "-save-vocab", v] + flag_args(golden), t)
        assert r.returncode == 0, r.stderr
        assert open(v, "rb").read() == open(os.path.join(golden.dir, "vocab.txt"), "rb").read()


def test_missing_file_fails_loudly():
    with tempfile.TemporaryDirectory() as t:
        r = run_cli(["-train", "/nonexistent", "-output", "o"], t)
        assert r.returncode != 0 and "parw2v:" in r.stderr


@pytest.mark.gpu
def test_det_mode_output_file_is_byte_identical(golden):
    if golden.output is None:
        pytest.skip("no reference output stored for this case")
    with tempfile.TemporaryDirectory() as t:
        out = os.path.join(t, "vectors.txt")
        r = run_cli(["-train", golden.corpus_path, "-output", out, "-mode", "det", "-binary", "0"] + flag_args(golden), t)
        assert r.returncode == 0, r.stderr
        assert open(out, "rb").read() == golden.output
        assert open(os.path.join(t, "PAR_Word2Vec_gpu_time")).read().startswith("Elapsed ")


@pytest.mark.gpu
def test_batched_mode_runs_and_writes_the_format(golden_cases):
    g = golden_cases["d100"]
    with tempfile.TemporaryDirectory() as t:
        out = os.path.join(t, "vectors.txt")
        r = run_cli(["-train", g.corpus_path, "-output", out, "-mode", "batched_bf16"] + flag_args(g), t)
        assert r.returncode == 0, r.stderr
        lines = open(out, "rb").read().split(b"\n")
        assert lines[0] == b"%d %d" % (len(g.words), int(g.flags["size"]))
        assert lines[1].split(b" ")[0] == g.words[0] and len(lines[1].split(b" ")) == int(g.flags["size"]) + 2
