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


def _adversarial_text(seed: int, n_lines: int) -> bytes:
    """Lines of words with every separator the tokenizer treats specially: carriage returns inside
    and between words, tabs, runs of spaces, blank lines, words past the 98-byte cut, repeated
    newlines, and no newline at the end of the file."""
    rng = np.random.default_rng(seed)
    alphabet = np.frombuffer(b"abcdefghij", dtype=np.uint8)
    lines = []
    for _ in range(n_lines):
        parts = []
        for _ in range(int(rng.integers(0, 30))):
            n = int(rng.choice([1, 2, 3, 5, 8, 120]))
            w = bytes(alphabet[rng.integers(0, 4 if n < 8 else 10, size=n)])
            if rng.random() < 0.05:
                w = w[: len(w) // 2] + b"\r" + w[len(w) // 2:]
            parts.append(w)
            parts.append([b" ", b"  ", b"\t", b" \r "][int(rng.integers(0, 4))])
        lines.append(b"".join(parts))
        if rng.random() < 0.1:
            lines.append(b"")
    return b"\n".join(lines) + b"\nlast words without newline"


@pytest.mark.parametrize("seed,n_lines", [(1, 40), (2, 4000)])
def test_threaded_front_end_matches_reference_on_many_ranges(seed, n_lines):
    """The front end cuts files into one byte range per host thread (ranges of 1 KB and up); on a
    text with every tokenizer edge case spread over many ranges the vocabulary must equal the
    reference binary's -save-vocab output byte for byte, and the stream the restated reader's."""
    from oracle import pwo, ref_text
    data = _adversarial_text(seed, n_lines)
    with tempfile.TemporaryDirectory() as t:
        corpus = os.path.join(t, "c.txt")
        open(corpus, "wb").write(data)
        v = pw.Vocab.learn(corpus, 1)
        ours = os.path.join(t, "ours.vocab")
        v.save(ours)
        stream = v.load_stream(corpus)
        want_stream = ref_text.stream_from_text(data, v.words())[:-1]
        assert np.array_equal(stream, want_stream)
        if not os.path.exists(pwo.REF_BIN):
            pytest.skip("reference not built (make -C oracle ref)")
        ref = os.path.join(t, "ref.vocab")
        # the reference also needs -output (with -save-vocab alone it crashes after saving nothing)
        subprocess.run([pwo.REF_BIN, "-train", corpus, "-save-vocab", ref, "-min-count", "1", "-debug", "0",
                        "-output", os.path.join(t, "o.bin"), "-binary", "1", "-size", "8", "-iter", "1",
                        "-threads", "1", "-window", "2", "-negative", "2", "-sample", "0"],
                       check=True, cwd=t, stdout=subprocess.DEVNULL)
        assert open(ours, "rb").read() == open(ref, "rb").read()
