import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")
CASES = ["text_small", "graph_small", "edge", "d100"]


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def gpu_available() -> bool:
    try:
        import ctypes
        rt = ctypes.CDLL("libcudart.so.12")
    except OSError:
        try:
            import torch  # only to locate a CUDA runtime when libcudart is not on the path
            return torch.cuda.is_available()
        except Exception:
            return False
    n = ctypes.c_int(0)
    return rt.cudaGetDeviceCount(ctypes.byref(n)) == 0 and n.value > 0


def pytest_collection_modifyitems(config, items):
    if gpu_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device visible")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


class Golden:
    def __init__(self, case: str):
        d = os.path.join(GOLDEN, case)
        self.case = case
        self.dir = d
        self.corpus_path = os.path.join(d, "corpus.txt")
        self.meta = json.load(open(os.path.join(d, "meta.json")))
        self.flags = self.meta["flags"]
        from oracle import ref_text
        self.words, self.counts = ref_text.load_vocab(os.path.join(d, "vocab.txt"))
        self.stream = ref_text.stream_from_text(open(self.corpus_path, "rb").read(), self.words)
        self.win = np.load(os.path.join(d, "win.npy"))
        self.wout = np.load(os.path.join(d, "wout.npy"))
        self.exptable = np.load(os.path.join(d, "exptable.npy"))
        out = os.path.join(d, "output.txt")
        self.output = open(out, "rb").read() if os.path.exists(out) else None

    def train_kwargs(self):
        f = self.flags
        return dict(size=int(f["size"]), window=int(f["window"]), negative=int(f["negative"]),
                    batch_size=int(f["batch_size"]), iter=int(f["iter"]), alpha=float(np.float32(f["alpha"])),
                    sample=float(np.float32(f["sample"])))


@pytest.fixture(scope="session", params=CASES)
def golden(request):
    return Golden(request.param)


@pytest.fixture(scope="session")
def golden_cases():
    return {c: Golden(c) for c in CASES}
