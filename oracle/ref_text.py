"""TEST INFRASTRUCTURE ONLY: the reference's text reader, restated in Python.

Used by tests/ and tests/golden/make_golden.py to turn a corpus file into the word-id
stream that the reference trains on, given the reference's vocabulary.

``ReadWord`` (PAR_Word2Vec_cpu.cpp:120-144) semantics, restated:
  * carriage returns (13) are skipped everywhere;
  * space, tab and newline end a word; a newline on its own is the word "</s>";
  * a word keeps at most its first 98 bytes (the ``a >= MAX_STRING - 1`` clamp);
  * a word still open at end of file is discarded by every caller (the caller sees
    ``feof`` after the read, :268-270 and :172-173);
  * a NUL byte ends the C string.
``loadStream`` (:359-370) maps words through the vocabulary, drops out-of-vocabulary
words and appends one "</s>" (id 0) sentinel.
"""
from __future__ import annotations

import re

import numpy as np

_TOKEN = re.compile(rb"[^ \t\n]+(?=[ \t\n])|\n")


def read_words(data: bytes) -> list[bytes]:
    data = data.replace(b"\r", b"")
    out = []
    for m in _TOKEN.finditer(data):
        t = m.group(0)
        if t == b"\n":
            out.append(b"</s>")
        else:
            out.append(t[:98].split(b"\0", 1)[0])
    return out


def load_vocab(path: str) -> tuple[list[bytes], np.ndarray]:
    """Read a ``word count`` per line vocabulary (the reference's -save-vocab format)."""
    words, counts = [], []
    with open(path, "rb") as f:
        for line in f:
            w, c = line.rstrip(b"\n").rsplit(b" ", 1)
            words.append(w)
            counts.append(int(c))
    return words, np.array(counts, dtype=np.uint32)


def stream_from_text(data: bytes, words: list[bytes]) -> np.ndarray:
    """Word ids of the corpus in file order (OOV dropped) plus the trailing 0 sentinel."""
    index = {w: i for i, w in enumerate(words)}
    ids = [index[w] for w in read_words(data) if w in index]
    ids.append(0)
    return np.array(ids, dtype=np.int32)
