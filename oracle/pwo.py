"""TEST INFRASTRUCTURE ONLY: ctypes wrapper of the C restatement (libparw2v_oracle.so).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this module, and
only as the checker.  Build with ``make -C oracle restatement``.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libparw2v_oracle.so")
REF_BIN = os.path.join(HERE, "_ref", "par_w2v_ref")
REF_FAST_BIN = os.path.join(HERE, "_ref", "par_w2v_ref_fast")
TABLE_SIZE = 100_000_000


class Config(ctypes.Structure):
    _fields_ = [("vocab_size", ctypes.c_int), ("hidden_size", ctypes.c_int), ("window", ctypes.c_int),
                ("negative", ctypes.c_int), ("batch_size", ctypes.c_int), ("iter", ctypes.c_int),
                ("alpha", ctypes.c_float), ("sample", ctypes.c_float), ("seed", ctypes.c_uint64),
                ("sync_window", ctypes.c_int)]


class Trace(ctypes.Structure):
    _fields_ = [("keep", ctypes.c_void_p), ("keep_cap", ctypes.c_int64), ("n_keep", ctypes.c_int64),
                ("b", ctypes.c_void_p), ("b_cap", ctypes.c_int64), ("n_b", ctypes.c_int64),
                ("alpha", ctypes.c_void_p), ("alpha_cap", ctypes.c_int64), ("n_alpha", ctypes.c_int64),
                ("rep_b", ctypes.c_void_p), ("rep_b_cap", ctypes.c_int64), ("n_rep_b", ctypes.c_int64),
                ("neg", ctypes.c_void_p), ("neg_cap", ctypes.c_int64), ("n_neg", ctypes.c_int64),
                ("n_pairs", ctypes.c_int64), ("n_sentences", ctypes.c_int64),
                ("words_read", ctypes.c_uint64), ("final_lcg", ctypes.c_uint64)]


_lib = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE, "restatement"], check=True)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        P = ctypes.c_void_p
        L.pwo_exp_table.argtypes = [P]
        L.pwo_unigram_table.argtypes = [P, ctypes.c_int, P]
        L.pwo_init_net.argtypes = [P, P, ctypes.c_int, ctypes.c_int]
        L.pwo_train.argtypes = [P, P, P, P, P, ctypes.c_uint64, P, P, P, ctypes.c_int64]
        L.pwo_train.restype = ctypes.c_int
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def exp_table() -> np.ndarray:
    out = np.zeros(1001, np.float32)
    lib().pwo_exp_table(_p(out))
    return out


def unigram_table(counts: np.ndarray) -> np.ndarray:
    c = np.ascontiguousarray(counts, np.uint32)
    out = np.empty(TABLE_SIZE, np.int32)
    lib().pwo_unigram_table(_p(c), len(c), _p(out))
    return out


def init_net(vocab_size: int, size: int):
    w_in = np.empty((vocab_size, size), np.float32)
    w_out = np.empty((vocab_size, size), np.float32)
    lib().pwo_init_net(_p(w_in), _p(w_out), vocab_size, size)
    return w_in, w_out


def train(counts, stream_with_sentinel, w_in, w_out, *, size, window, negative, batch_size, iter, alpha, sample,
          seed=0, table=None, trace_caps=None, max_resample=0, sync_window=0):
    """Run the restated loop in place on w_in / w_out; returns the trace dict."""
    c = np.ascontiguousarray(counts, np.uint32)
    s = np.ascontiguousarray(stream_with_sentinel, np.int32)
    if table is None:
        table = unigram_table(c)
    et = exp_table()
    cfg = Config(len(c), size, window, negative, batch_size, iter, alpha, sample, seed, int(sync_window))
    caps = trace_caps or {}
    bufs = dict(keep=np.zeros(caps.get("keep", 0), np.uint8), b=np.zeros(caps.get("b", 0), np.uint8),
                alpha=np.zeros(caps.get("alpha", 0), np.float32), rep_b=np.zeros(caps.get("rep_b", 0), np.uint8),
                neg=np.zeros(caps.get("neg", 0), np.int32))
    tr = Trace()
    for k, v in bufs.items():
        setattr(tr, k, v.ctypes.data if len(v) else None)
        setattr(tr, k + "_cap", len(v))
    rc = lib().pwo_train(ctypes.byref(cfg), _p(c), _p(table), _p(et), _p(s), len(s) - 1, _p(w_in), _p(w_out),
                         ctypes.byref(tr), int(max_resample))
    out = {k: v[: min(len(v), getattr(tr, "n_" + k))] for k, v in bufs.items()}
    out.update({"n_" + k: int(getattr(tr, "n_" + k)) for k in bufs})
    out.update(rc=rc, n_pairs=tr.n_pairs, n_sentences=tr.n_sentences, words_read=tr.words_read,
               final_lcg=tr.final_lcg)
    return out
