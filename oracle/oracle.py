"""ctypes front end of the CPU oracle (test infrastructure only).

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module; the product path never does.  The C code it
loads (``oracle/bt_oracle.c``) restates the reference's B+tree rules and batch
semantics; every function there cites the reference file:line it follows.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

OP_INSERT = 0
OP_GET = 1
OP_DELETE = 2
ABSENT, FOUND, REJECTED = 0, 1, 2
ENGINE_STM, ENGINE_MERGE = 0, 1
DIST = {"uniform": 0, "zipf": 1, "normal": 2, "gamma": 3}

_u64p = ctypes.POINTER(ctypes.c_uint64)
_u32p = ctypes.POINTER(ctypes.c_uint32)
_u8p = ctypes.POINTER(ctypes.c_uint8)
_f32p = ctypes.POINTER(ctypes.c_float)
_f64p = ctypes.POINTER(ctypes.c_double)


class Stats(ctypes.Structure):
    _fields_ = [
        ("n_keys", ctypes.c_uint64),
        ("n_nodes", ctypes.c_uint64),
        ("n_leaves", ctypes.c_uint64),
        ("height", ctypes.c_uint32),
        ("root_level", ctypes.c_uint32),
        ("leaf_splits", ctypes.c_uint64),
        ("inner_splits", ctypes.c_uint64),
        ("new_roots", ctypes.c_uint64),
    ]


def build() -> str:
    """Compile liboracle.so in place (gcc only)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(
            os.path.join(HERE, "bt_oracle.c")
        ):
            build()
        L = ctypes.CDLL(LIB_PATH)
        L.bto_create.restype = ctypes.c_void_p
        L.bto_create.argtypes = [ctypes.c_uint32, ctypes.c_uint32]
        L.bto_destroy.argtypes = [ctypes.c_void_p]
        L.bto_bulk_build.argtypes = [ctypes.c_void_p, _u64p, _u64p, ctypes.c_size_t]
        L.bto_get.argtypes = [ctypes.c_void_p, ctypes.c_uint64, _u64p]
        L.bto_insert.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64, _u64p]
        L.bto_execute_serial.argtypes = [ctypes.c_void_p, _u64p, _u64p, _u8p, ctypes.c_size_t, _u64p, _u8p]
        L.bto_execute_merged.argtypes = [
            ctypes.c_void_p, _u64p, _u64p, _u8p, ctypes.c_size_t, _u64p, _u8p, ctypes.c_int, ctypes.c_int,
        ]
        L.bto_size.restype = ctypes.c_size_t
        L.bto_size.argtypes = [ctypes.c_void_p]
        L.bto_dump.argtypes = [ctypes.c_void_p, _u64p, _u64p]
        L.bto_leaf_sizes.restype = ctypes.c_size_t
        L.bto_leaf_sizes.argtypes = [ctypes.c_void_p, _u32p, ctypes.c_size_t]
        L.bto_leaf_lows.restype = ctypes.c_size_t
        L.bto_leaf_lows.argtypes = [ctypes.c_void_p, _u64p, ctypes.c_size_t]
        L.bto_level_counts.restype = ctypes.c_uint32
        L.bto_level_counts.argtypes = [ctypes.c_void_p, _u64p, ctypes.c_uint32]
        L.bto_get_stats.argtypes = [ctypes.c_void_p, ctypes.POINTER(Stats)]
        L.bto_check.argtypes = [ctypes.c_void_p]
        L.bto_sort_pairs.argtypes = [_u64p, ctypes.c_size_t, _u64p, _u32p]
        L.bto_mlp_forward.restype = ctypes.c_double
        L.bto_mlp_forward.argtypes = [_f32p, ctypes.c_double]
        L.bto_mlp_grad.restype = ctypes.c_double
        L.bto_mlp_grad.argtypes = [_f32p, _f32p, _f32p, ctypes.c_size_t, _f64p]
        L.bto_mix64.restype = ctypes.c_uint64
        L.bto_mix64.argtypes = [ctypes.c_uint64]
        L.bto_gen_keys.argtypes = [ctypes.c_int, ctypes.c_uint64, ctypes.c_size_t, _u64p]
        L.bto_value_of.restype = ctypes.c_uint64
        L.bto_value_of.argtypes = [ctypes.c_uint64]
        L.bto_gen_requests.argtypes = [
            ctypes.c_int, ctypes.c_uint64, _u64p, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_uint32,
            _u64p, _u64p, _u8p,
        ]
        _lib = L
    return _lib


def _p(a: np.ndarray, t):
    return a.ctypes.data_as(t)


def _u64(a):
    return np.ascontiguousarray(a, dtype=np.uint64)


class OracleTree:
    """CPU restatement of the reference tree (one object = one tree)."""

    def __init__(self, leaf_fill: int = 24, inner_fill: int = 24):
        self._h = lib().bto_create(leaf_fill, inner_fill)
        self.leaf_fill, self.inner_fill = leaf_fill, inner_fill

    def __del__(self):
        if getattr(self, "_h", None):
            try:
                lib().bto_destroy(self._h)
            except Exception:  # interpreter shutdown: the module globals are gone
                pass
            self._h = None

    def bulk_build(self, keys, vals):
        k, v = _u64(keys), _u64(vals)
        rc = lib().bto_bulk_build(self._h, _p(k, _u64p), _p(v, _u64p), k.size)
        if rc != 0:
            raise ValueError("reserved key in bulk build")

    def get(self, key: int):
        v = ctypes.c_uint64(0)
        st = lib().bto_get(self._h, key, ctypes.byref(v))
        return st, v.value

    def insert(self, key: int, val: int):
        v = ctypes.c_uint64(0)
        st = lib().bto_insert(self._h, key, val, ctypes.byref(v))
        return st, v.value

    def execute_serial(self, keys, vals, ops):
        k, v, o = _u64(keys), _u64(vals), np.ascontiguousarray(ops, dtype=np.uint8)
        ov = np.zeros(k.size, np.uint64)
        os_ = np.zeros(k.size, np.uint8)
        lib().bto_execute_serial(self._h, _p(k, _u64p), _p(v, _u64p), _p(o, _u8p), k.size,
                                 _p(ov, _u64p), _p(os_, _u8p))
        return ov, os_

    def execute_merged(self, keys, vals, ops, engine=ENGINE_STM, threads=1):
        k, v, o = _u64(keys), _u64(vals), np.ascontiguousarray(ops, dtype=np.uint8)
        ov = np.zeros(k.size, np.uint64)
        os_ = np.zeros(k.size, np.uint8)
        lib().bto_execute_merged(self._h, _p(k, _u64p), _p(v, _u64p), _p(o, _u8p), k.size,
                                 _p(ov, _u64p), _p(os_, _u8p), engine, threads)
        return ov, os_

    def size(self) -> int:
        return lib().bto_size(self._h)

    def dump(self):
        n = self.size()
        k = np.zeros(n, np.uint64)
        v = np.zeros(n, np.uint64)
        lib().bto_dump(self._h, _p(k, _u64p), _p(v, _u64p))
        return k, v

    def leaf_sizes(self):
        n = lib().bto_leaf_sizes(self._h, None, 0)
        s = np.zeros(n, np.uint32)
        lib().bto_leaf_sizes(self._h, _p(s, _u32p), n)
        return s

    def leaf_lows(self):
        n = lib().bto_leaf_lows(self._h, None, 0)
        s = np.zeros(n, np.uint64)
        lib().bto_leaf_lows(self._h, _p(s, _u64p), n)
        return s

    def level_counts(self):
        c = np.zeros(32, np.uint64)
        h = lib().bto_level_counts(self._h, _p(c, _u64p), 32)
        return c[:h]

    def stats(self) -> dict:
        s = Stats()
        lib().bto_get_stats(self._h, ctypes.byref(s))
        return {f: getattr(s, f) for f, _ in Stats._fields_}

    def check(self) -> int:
        return lib().bto_check(self._h)


def sort_pairs(keys):
    k = _u64(keys)
    ko = np.zeros(k.size, np.uint64)
    io = np.zeros(k.size, np.uint32)
    lib().bto_sort_pairs(_p(k, _u64p), k.size, _p(ko, _u64p), _p(io, _u32p))
    return ko, io


def gen_keys(dist: str, seed: int, n: int):
    k = np.zeros(n, np.uint64)
    lib().bto_gen_keys(DIST[dist], seed, n, _p(k, _u64p))
    return k


def value_of(keys):
    return _u64(keys) ^ np.uint64(0x9E3779B97F4A7C15)


def gen_requests(dist: str, seed: int, tree_keys, n: int, search_pct: int):
    tk = _u64(tree_keys)
    k = np.zeros(n, np.uint64)
    v = np.zeros(n, np.uint64)
    o = np.zeros(n, np.uint8)
    lib().bto_gen_requests(DIST[dist], seed, _p(tk, _u64p), tk.size, n, search_pct,
                           _p(k, _u64p), _p(v, _u64p), _p(o, _u8p))
    return k, v, o


def mlp_forward(params, x: float) -> float:
    p = np.ascontiguousarray(params, dtype=np.float32)
    return lib().bto_mlp_forward(_p(p, _f32p), float(x))


def mlp_grad(params, x, y):
    p = np.ascontiguousarray(params, dtype=np.float32)
    xs = np.ascontiguousarray(x, dtype=np.float32)
    ys = np.ascontiguousarray(y, dtype=np.float32)
    g = np.zeros(97, np.float64)
    loss = lib().bto_mlp_grad(_p(p, _f32p), _p(xs, _f32p), _p(ys, _f32p), xs.size, _p(g, _f64p))
    return loss, g
