"""B200-native PAR-Word2Vec: Python host bindings over the C ABI of ``libparw2v.so``.

The reference (gordonmoon/PAR_Word2Vec) is driven by its command line; the library behind
``include/parw2v.h`` replaces ``Train_PAR_Word2Vec`` (PAR_Word2Vec_cpu.cpp:372-711,
PAR_Word2Vec_gpu_text.cu:726-979) and its text front end.  This module is a thin ctypes
mirror of that ABI; every call goes to the CUDA library and raises ``ParW2VError`` on a
non-zero status.  There is no CPU fallback: without the built library (or without a GPU for
device calls) the calls fail loudly.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

__all__ = ["ParW2VError", "Config", "Trainer", "Vocab", "load_library", "MODE_DET", "MODE_PLAIN",
           "MODE_BATCHED", "MODE_BATCHED_BF16", "TABLE_SIZE", "EXP_TABLE_SIZE", "LIB_PATH"]

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libparw2v.so")
MODE_DET, MODE_PLAIN, MODE_BATCHED, MODE_BATCHED_BF16 = 0, 1, 2, 3
MODE_NAMES = {"det": MODE_DET, "plain": MODE_PLAIN, "batched": MODE_BATCHED, "batched_bf16": MODE_BATCHED_BF16}
TABLE_SIZE = 100_000_000
EXP_TABLE_SIZE = 1000

ATTRACT_DEFAULT, ATTRACT_SEQUENTIAL, ATTRACT_WINDOW, ATTRACT_PIPELINED = 0, 1, 2, 3
VARIANT_AUTO, VARIANT_WINDOW, VARIANT_STREAM = 0, 1, 2
STAGING_AUTO, STAGING_BULK, STAGING_CPASYNC = 0, 1, 2
REPULSION_SERIAL, REPULSION_TENSOR, REPULSION_CUDA = 0, 1, 2
OK, ERR_ARG, ERR_CUDA, ERR_OOM, ERR_CAPACITY, ERR_TIMEOUT, ERR_STATE, ERR_IO, ERR_NODEV = 0, -1, -2, -3, -4, -5, -6, -7, -8

# every symbol include/parw2v.h declares (checked by tests against the built library)
EXPORTED = [
    "parw2v_version", "parw2v_strerror", "parw2v_last_error", "parw2v_create", "parw2v_destroy",
    "parw2v_set_vocab", "parw2v_get_table", "parw2v_get_exp_table", "parw2v_init_weights",
    "parw2v_set_weights", "parw2v_get_weights", "parw2v_set_corpus", "parw2v_train", "parw2v_set_trace",
    "parw2v_loss", "parw2v_loss_adjoint", "parw2v_loss_fd", "parw2v_vocab_learn", "parw2v_vocab_read",
    "parw2v_vocab_free", "parw2v_vocab_size", "parw2v_vocab_train_words", "parw2v_vocab_counts",
    "parw2v_vocab_word", "parw2v_vocab_save", "parw2v_load_stream", "parw2v_save_model",
    "parw2v_det_train_noalloc", "parw2v_random_walks",
]


class ParW2VError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"parw2v error {status}: {message}")
        self.status = status


class Config(ctypes.Structure):
    _fields_ = [("size", ctypes.c_int), ("window", ctypes.c_int), ("negative", ctypes.c_int),
                ("batch_size", ctypes.c_int), ("iter", ctypes.c_int), ("alpha", ctypes.c_float),
                ("sample", ctypes.c_float), ("mode", ctypes.c_int), ("device", ctypes.c_int),
                ("seed", ctypes.c_uint64), ("grid", ctypes.c_int), ("warps_per_cta", ctypes.c_int),
                ("mem_cap_bytes", ctypes.c_size_t), ("min_rounds", ctypes.c_int), ("attraction", ctypes.c_int),
                ("variant", ctypes.c_int), ("staging", ctypes.c_int), ("autotune", ctypes.c_int)]


class _Stats(ctypes.Structure):
    _fields_ = [("words", ctypes.c_uint64), ("kept", ctypes.c_uint64), ("sentences", ctypes.c_uint64),
                ("pairs", ctypes.c_uint64), ("batches", ctypes.c_uint64), ("negatives", ctypes.c_uint64),
                ("kernel_ms", ctypes.c_double), ("pack_ms", ctypes.c_double), ("final_alpha", ctypes.c_float),
                ("grid", ctypes.c_int), ("warps_per_cta", ctypes.c_int), ("repulsion", ctypes.c_int),
                ("lane_elems", ctypes.c_int), ("staging", ctypes.c_int), ("attraction", ctypes.c_int),
                ("variant", ctypes.c_int)]


class _Trace(ctypes.Structure):
    _fields_ = [("keep", ctypes.c_void_p), ("keep_cap", ctypes.c_int64), ("n_keep", ctypes.c_int64),
                ("b", ctypes.c_void_p), ("b_cap", ctypes.c_int64), ("n_b", ctypes.c_int64),
                ("alpha", ctypes.c_void_p), ("alpha_cap", ctypes.c_int64), ("n_alpha", ctypes.c_int64),
                ("rep_b", ctypes.c_void_p), ("rep_b_cap", ctypes.c_int64), ("n_rep_b", ctypes.c_int64),
                ("neg", ctypes.c_void_p), ("neg_cap", ctypes.c_int64), ("n_neg", ctypes.c_int64),
                ("final_lcg", ctypes.c_uint64)]


_lib = None


def load_library(path: str = LIB_PATH) -> ctypes.CDLL:
    """Load libparw2v.so (built by ``python -m par_word2vec_b200.build``)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ParW2VError(ERR_NODEV, f"{path} is not built; run python -m par_word2vec_b200.build")
    lib = ctypes.CDLL(path)
    P, I, U64, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_uint64, ctypes.c_double
    sig = {
        "parw2v_version": ([], ctypes.c_char_p), "parw2v_strerror": ([I], ctypes.c_char_p),
        "parw2v_last_error": ([P], ctypes.c_char_p), "parw2v_create": ([P, P], I),
        "parw2v_destroy": ([P], None), "parw2v_set_vocab": ([P, P, I], I), "parw2v_get_table": ([P, P], I),
        "parw2v_get_exp_table": ([P, P], I), "parw2v_init_weights": ([P], I),
        "parw2v_set_weights": ([P, P, P], I), "parw2v_get_weights": ([P, P, P], I),
        "parw2v_set_corpus": ([P, P, U64], I), "parw2v_train": ([P, P], I), "parw2v_set_trace": ([P, P], I),
        "parw2v_loss": ([P, P, P, I, P, I, I, P], I),
        "parw2v_loss_adjoint": ([P, P, P, I, P, I, I, I, P, P], I),
        "parw2v_loss_fd": ([P, P, P, I, P, I, I, P, P, P, I, D, P], I),
        "parw2v_vocab_learn": ([ctypes.c_char_p, I, P], I), "parw2v_vocab_read": ([ctypes.c_char_p, I, P], I),
        "parw2v_vocab_free": ([P], None), "parw2v_vocab_size": ([P], I), "parw2v_vocab_train_words": ([P], U64),
        "parw2v_vocab_counts": ([P, P], I), "parw2v_vocab_word": ([P, I], ctypes.c_char_p),
        "parw2v_vocab_save": ([P, ctypes.c_char_p], I),
        "parw2v_load_stream": ([P, ctypes.c_char_p, P, U64, P], I),
        "parw2v_save_model": ([P, P, I, I, ctypes.c_char_p], I),
        "parw2v_det_train_noalloc": ([P, I, U64, P, U64, P, P, P, P, P, I, P, P], I),
        "parw2v_random_walks": ([P, P, I, I, I, U64, I, P], I),
    }
    for name, (args, res) in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


class Vocab:
    """The reference's vocabulary (LearnVocabFromTrainFile / ReadVocab + SortVocab)."""

    def __init__(self, handle):
        self._h = handle
        self._lib = load_library()

    @classmethod
    def learn(cls, train_file: str, min_count: int = 5) -> "Vocab":
        lib = load_library()
        h = ctypes.c_void_p()
        rc = lib.parw2v_vocab_learn(train_file.encode(), int(min_count), ctypes.byref(h))
        if rc:
            raise ParW2VError(rc, f"cannot learn vocabulary from {train_file}")
        return cls(h)

    @classmethod
    def read(cls, vocab_file: str, min_count: int = 5) -> "Vocab":
        lib = load_library()
        h = ctypes.c_void_p()
        rc = lib.parw2v_vocab_read(vocab_file.encode(), int(min_count), ctypes.byref(h))
        if rc:
            raise ParW2VError(rc, f"cannot read vocabulary {vocab_file}")
        return cls(h)

    def __del__(self):
        if getattr(self, "_h", None):
            self._lib.parw2v_vocab_free(self._h)
            self._h = None

    def __len__(self) -> int:
        return self._lib.parw2v_vocab_size(self._h)

    @property
    def train_words(self) -> int:
        return int(self._lib.parw2v_vocab_train_words(self._h))

    def counts(self) -> np.ndarray:
        out = np.zeros(len(self), dtype=np.uint32)
        self._lib.parw2v_vocab_counts(self._h, _ptr(out))
        return out

    def words(self) -> list[bytes]:
        return [self._lib.parw2v_vocab_word(self._h, i) for i in range(len(self))]

    def save(self, path: str) -> None:
        rc = self._lib.parw2v_vocab_save(self._h, path.encode())
        if rc:
            raise ParW2VError(rc, f"cannot write {path}")

    def load_stream(self, train_file: str) -> np.ndarray:
        # loadStream keeps at most train_words ids, so one pass into a buffer of that size suffices
        n = ctypes.c_uint64()
        cap = max(1, self.train_words)
        out = np.zeros(cap, dtype=np.int32)
        rc = self._lib.parw2v_load_stream(self._h, train_file.encode(), _ptr(out), cap, ctypes.byref(n))
        if rc:
            raise ParW2VError(rc, f"cannot read {train_file}")
        return out[: n.value]

    def save_model(self, w_in: np.ndarray, path: str, binary: bool = False) -> None:
        w = np.ascontiguousarray(w_in, dtype=np.float32)
        rc = self._lib.parw2v_save_model(self._h, _ptr(w), int(w.shape[1]), int(bool(binary)), path.encode())
        if rc:
            raise ParW2VError(rc, f"cannot write {path}")


class Trainer:
    """One training context on one CUDA device (``parw2v_create`` .. ``parw2v_destroy``)."""

    def __init__(self, size=100, window=5, negative=5, batch_size=24, iter=5, alpha=0.025, sample=1e-3,
                 mode=MODE_BATCHED_BF16, device=0, seed=0, grid=0, warps_per_cta=0, mem_cap_bytes=0, min_rounds=0, attraction=0,
                 variant=0, staging=0, autotune=0):
        self._lib = load_library()
        if isinstance(mode, str):
            mode = MODE_NAMES[mode]
        self.cfg = Config(int(size), int(window), int(negative), int(batch_size), int(iter), float(alpha),
                          float(sample), int(mode), int(device), int(seed), int(grid), int(warps_per_cta),
                          int(mem_cap_bytes), int(min_rounds), int(attraction), int(variant), int(staging),
                          int(autotune))
        self._h = ctypes.c_void_p()
        rc = self._lib.parw2v_create(ctypes.byref(self.cfg), ctypes.byref(self._h))
        if rc:
            raise ParW2VError(rc, self._lib.parw2v_last_error(None).decode())
        self.vocab_size = 0
        self._trace = None

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.parw2v_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc: int) -> None:
        if rc:
            raise ParW2VError(rc, self._lib.parw2v_last_error(self._h).decode())

    @property
    def size(self) -> int:
        return self.cfg.size

    def set_vocab(self, counts) -> None:
        c = np.ascontiguousarray(counts, dtype=np.uint32)
        self._check(self._lib.parw2v_set_vocab(self._h, _ptr(c), int(len(c))))
        self.vocab_size = len(c)

    def get_table(self) -> np.ndarray:
        out = np.empty(TABLE_SIZE, dtype=np.int32)
        self._check(self._lib.parw2v_get_table(self._h, _ptr(out)))
        return out

    def get_exp_table(self) -> np.ndarray:
        out = np.empty(EXP_TABLE_SIZE + 1, dtype=np.float32)
        self._check(self._lib.parw2v_get_exp_table(self._h, _ptr(out)))
        return out

    def init_weights(self) -> None:
        self._check(self._lib.parw2v_init_weights(self._h))

    def set_weights(self, w_in=None, w_out=None) -> None:
        a = None if w_in is None else np.ascontiguousarray(w_in, dtype=np.float32)
        b = None if w_out is None else np.ascontiguousarray(w_out, dtype=np.float32)
        self._check(self._lib.parw2v_set_weights(self._h, _ptr(a), _ptr(b)))

    def get_weights(self, which: str = "both"):
        shape = (self.vocab_size, self.cfg.size)
        a = np.empty(shape, dtype=np.float32) if which in ("both", "in") else None
        b = np.empty(shape, dtype=np.float32) if which in ("both", "out") else None
        self._check(self._lib.parw2v_get_weights(self._h, _ptr(a), _ptr(b)))
        return (a, b) if which == "both" else (a if which == "in" else b)

    def set_corpus(self, tokens) -> None:
        t = np.ascontiguousarray(tokens, dtype=np.int32)
        self._check(self._lib.parw2v_set_corpus(self._h, _ptr(t), int(len(t))))

    def set_trace(self, keep_cap=0, b_cap=0, alpha_cap=0, rep_b_cap=0, neg_cap=0) -> None:
        bufs = dict(keep=np.zeros(keep_cap, np.uint8), b=np.zeros(b_cap, np.uint8),
                    alpha=np.zeros(alpha_cap, np.float32), rep_b=np.zeros(rep_b_cap, np.uint8),
                    neg=np.zeros(neg_cap, np.int32))
        t = _Trace()
        for k, v in bufs.items():
            setattr(t, k, v.ctypes.data if len(v) else None)
            setattr(t, k + "_cap", len(v))
        self._trace = (t, bufs)
        self._check(self._lib.parw2v_set_trace(self._h, ctypes.byref(t)))

    def trace(self) -> dict:
        t, bufs = self._trace
        out = {k: v[: min(len(v), getattr(t, "n_" + k))] for k, v in bufs.items()}
        out.update({"n_" + k: int(getattr(t, "n_" + k)) for k in bufs})
        out["final_lcg"] = int(t.final_lcg)
        return out

    def train(self) -> dict:
        st = _Stats()
        self._check(self._lib.parw2v_train(self._h, ctypes.byref(st)))
        return {k: getattr(st, k) for k, _ in _Stats._fields_}

    def _batch(self, tgt, ctx, neg):
        t = np.ascontiguousarray(tgt, dtype=np.int32)
        c = np.ascontiguousarray(ctx, dtype=np.int32)
        n = np.ascontiguousarray(neg, dtype=np.int32)
        return t, c, n

    def loss(self, tgt, ctx, neg, n_neg: int, ctx_per_window: int) -> float:
        t, c, n = self._batch(tgt, ctx, neg)
        out = ctypes.c_double()
        self._check(self._lib.parw2v_loss(self._h, _ptr(t), _ptr(c), len(t), _ptr(n), int(n_neg),
                                          int(ctx_per_window), ctypes.byref(out)))
        return out.value

    def loss_adjoint(self, tgt, ctx, neg, n_neg: int, ctx_per_window: int, exact: bool = True):
        t, c, n = self._batch(tgt, ctx, neg)
        gi = np.empty((self.vocab_size, self.cfg.size), np.float32)
        go = np.empty((self.vocab_size, self.cfg.size), np.float32)
        self._check(self._lib.parw2v_loss_adjoint(self._h, _ptr(t), _ptr(c), len(t), _ptr(n), int(n_neg),
                                                  int(ctx_per_window), int(bool(exact)), _ptr(gi), _ptr(go)))
        return gi, go

    def loss_fd(self, tgt, ctx, neg, n_neg: int, ctx_per_window: int, matrix, row, col, h: float = 1e-3):
        t, c, n = self._batch(tgt, ctx, neg)
        m = np.ascontiguousarray(matrix, np.int32)
        r = np.ascontiguousarray(row, np.int32)
        k = np.ascontiguousarray(col, np.int32)
        out = np.empty(len(m), np.float64)
        self._check(self._lib.parw2v_loss_fd(self._h, _ptr(t), _ptr(c), len(t), _ptr(n), int(n_neg),
                                             int(ctx_per_window), _ptr(m), _ptr(r), _ptr(k), len(m), float(h),
                                             _ptr(out)))
        return out


def random_walks(indptr, indices, walks_per_node: int, walk_len: int, seed: int = 0, device: int = 0) -> np.ndarray:
    """Uniform random walks over a CSR graph on the GPU (``parw2v_random_walks``): an array of
    shape (walks_per_node * n_nodes, walk_len); walk w starts at node w mod n_nodes."""
    lib = load_library()
    ip = np.ascontiguousarray(indptr, dtype=np.int64)
    ix = np.ascontiguousarray(indices, dtype=np.int32)
    n = len(ip) - 1
    out = np.empty((walks_per_node * n, walk_len), dtype=np.int32)
    rc = lib.parw2v_random_walks(_ptr(ip), _ptr(ix), n, int(walks_per_node), int(walk_len), int(seed), int(device),
                                 _ptr(out))
    if rc:
        raise ParW2VError(rc, lib.parw2v_last_error(None).decode())
    return out
