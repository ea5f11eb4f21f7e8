"""Host front end of libparw2v (no GPU): the reference's tokenizer, vocabulary order, stream and
output format, checked against the reference's own outputs (tests/golden)."""
import ctypes
import os
import subprocess
import tempfile

import numpy as np
import pytest

import par_word2vec_b200 as pw
from tests.conftest import ROOT


def test_library_exports_every_declared_symbol():
    lib = pw.load_library()
    header = open(os.path.join(ROOT, "include", "parw2v.h")).read()
    declared = set()
    import re
    for m in re.finditer(r"\b(parw2v_[a-z_0-9]+)\s*\(", header):
        declared.add(m.group(1))
    assert declared == set(pw.EXPORTED)
    out = subprocess.run(["nm", "-D", "--defined-only", pw.LIB_PATH], capture_output=True, text=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if ln.strip()}
    missing = declared - exported
    assert not missing, missing
    for name in declared:
        assert getattr(lib, name) is not None


def test_version_and_errors():
    lib = pw.load_library()
    assert b"sm_100a" in lib.parw2v_version()
    assert lib.parw2v_strerror(pw.ERR_TIMEOUT) == b"bounded device loop gave up"
    assert lib.parw2v_strerror(12345) == b"unknown status"


def test_vocab_matches_reference(golden):
    v = pw.Vocab.learn(golden.corpus_path, int(golden.flags["min_count"]))
    assert v.words() == golden.words
    assert np.array_equal(v.counts(), golden.counts)
    assert v.train_words == golden.meta["train_words"]


def test_stream_matches_reference(golden):
    v = pw.Vocab.learn(golden.corpus_path, int(golden.flags["min_count"]))
    s = v.load_stream(golden.corpus_path)
    assert np.array_equal(s, golden.stream[:-1])


def test_save_model_is_byte_identical(golden):
    if golden.output is None:
        pytest.skip("no reference output stored for this case")
    v = pw.Vocab.learn(golden.corpus_path, int(golden.flags["min_count"]))
    with tempfile.TemporaryDirectory() as t:
        p = os.path.join(t, "o.txt")
        v.save_model(golden.win, p)
        assert open(p, "rb").read() == golden.output


def test_save_and_read_vocab_roundtrip(golden):
    v = pw.Vocab.learn(golden.corpus_path, int(golden.flags["min_count"]))
    with tempfile.TemporaryDirectory() as t:
        p = os.path.join(t, "v.txt")
        v.save(p)
        assert open(p, "rb").read() == open(os.path.join(golden.dir, "vocab.txt"), "rb").read()
        r = pw.Vocab.read(p, int(golden.flags["min_count"]))
        assert r.words() == golden.words and np.array_equal(r.counts(), golden.counts)


def test_binary_model_format(golden_cases):
    g = golden_cases["edge"]
    v = pw.Vocab.learn(g.corpus_path, int(g.flags["min_count"]))
    with tempfile.TemporaryDirectory() as t:
        p = os.path.join(t, "o.bin")
        v.save_model(g.win, p, binary=True)
        data = open(p, "rb").read()
    head, rest = data.split(b"\n", 1)
    assert head == b"%d %d" % g.win.shape
    off = 0
    for i, w in enumerate(g.words):
        assert rest[off: off + len(w) + 1] == w + b" "
        off += len(w) + 1
        row = np.frombuffer(rest[off: off + 4 * g.win.shape[1]], np.float32)
        assert np.array_equal(row.view(np.uint32), g.win[i].view(np.uint32))
        off += 4 * g.win.shape[1] + 1


def test_missing_file_is_an_error_not_an_exit():
    with pytest.raises(pw.ParW2VError) as e:
        pw.Vocab.learn("/nonexistent/corpus.txt")
    assert e.value.status == pw.ERR_IO


def test_empty_corpus():
    with tempfile.TemporaryDirectory() as t:
        p = os.path.join(t, "empty.txt")
        open(p, "wb").close()
        v = pw.Vocab.learn(p, 1)
        assert v.words() == [b"</s>"] and v.train_words == 0
        assert len(v.load_stream(p)) == 0
