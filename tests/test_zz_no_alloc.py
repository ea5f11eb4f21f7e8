"""parw2v_det_train_noalloc: deterministic training for callers that cannot let a library allocate
device memory (a framework whose caching allocator owns the GPU, or a service that reserves its
memory once at start-up).  The test owns every device buffer (allocated here with torch, as such a
caller would with its own allocator), calls the entry point through the C ABI twice in a row, and
checks each result against parw2v_train in DET mode with the DET tests' tolerance: bit-exact.
The second call also shows that what the first call left in the shared static scratch does not
leak into the next result."""
import ctypes

import numpy as np
import pytest

import par_word2vec_b200 as pw
from oracle import pwo

pytestmark = pytest.mark.gpu


def keep_thresholds(counts, sample, train_words):
    """sqrtf(r) + r with r = (sample * (float) train_words) / (float) count, all in FP32."""
    c = counts.astype(np.float32)
    with np.errstate(divide="ignore"):
        r = (np.float32(sample) * np.float32(train_words)) / c
    return (np.sqrt(r) + r).astype(np.float32)


def config(k, device=0):
    cfg = pw.Config()
    cfg.size, cfg.window, cfg.negative = k["size"], k["window"], k["negative"]
    cfg.batch_size, cfg.iter, cfg.alpha, cfg.sample = k["batch_size"], k["iter"], k["alpha"], k["sample"]
    cfg.mode, cfg.device, cfg.seed = pw.MODE_DET, device, 0
    return cfg


@pytest.mark.parametrize("case", ["text_small", "d100"])
def test_noalloc_matches_det_entry_point_on_two_calls(golden_cases, case):
    import torch

    g = golden_cases[case]
    k = g.train_kwargs()
    V, d = len(g.counts), k["size"]
    with pw.Trainer(mode=pw.MODE_DET, seed=0, **k) as t:  # the existing entry point
        t.set_vocab(g.counts)
        table, exp_table = t.get_table(), t.get_exp_table()
        t.init_weights()
        t.set_corpus(g.stream[:-1])
        t.train()
        want_in, want_out = t.get_weights()
    w0_in, _ = pwo.init_net(V, d)
    dev = torch.device("cuda:0")
    d_corpus = torch.from_numpy(g.stream.astype(np.int32)).to(dev)  # ids + the trailing 0
    d_table = torch.from_numpy(table).to(dev)
    d_exp = torch.from_numpy(exp_table).to(dev)
    d_thr = torch.from_numpy(keep_thresholds(g.counts, k["sample"], int(g.counts.sum()))).to(dev)
    lib = pw.load_library()
    cfg = config(k)
    for call in range(2):
        d_in = torch.from_numpy(w0_in).to(dev)
        d_out = torch.zeros((V, d), dtype=torch.float32, device=dev)
        st = pw._Stats()  # the library's parw2v_stats layout
        rc = lib.parw2v_det_train_noalloc(ctypes.byref(cfg), V, int(g.counts.sum()), d_corpus.data_ptr(),
                                          len(g.stream) - 1, d_table.data_ptr(), d_exp.data_ptr(),
                                          d_thr.data_ptr(), d_in.data_ptr(), d_out.data_ptr(), d,
                                          None, ctypes.byref(st))
        assert rc == 0, lib.parw2v_last_error(None)
        got_in, got_out = d_in.cpu().numpy(), d_out.cpu().numpy()
        assert np.array_equal(got_in.view(np.uint32), want_in.view(np.uint32)), f"call {call}: W_in differs"
        assert np.array_equal(got_out.view(np.uint32), want_out.view(np.uint32)), f"call {call}: W_out differs"
        assert st.words == k["iter"] * len(g.stream)


def test_noalloc_rejects_sizes_beyond_its_scratch(golden_cases):
    import torch

    g = golden_cases["edge"]
    k = dict(g.train_kwargs())
    k.update(size=4096, window=100, negative=100, batch_size=24)  # far beyond 1 MiB of staging rows
    cfg = config(k)
    lib = pw.load_library()
    dummy = torch.zeros(16, dtype=torch.int32, device="cuda:0")
    w = torch.zeros((len(g.counts), 4096), dtype=torch.float32, device="cuda:0")
    rc = lib.parw2v_det_train_noalloc(ctypes.byref(cfg), len(g.counts), int(g.counts.sum()), dummy.data_ptr(), 0,
                                      dummy.data_ptr(), dummy.data_ptr(), dummy.data_ptr(), w.data_ptr(),
                                      w.data_ptr(), 4096, None, None)
    assert rc == pw.ERR_CAPACITY
    assert b"1 MiB" in lib.parw2v_last_error(None)
