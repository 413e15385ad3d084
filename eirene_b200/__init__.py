"""eirene_b200: B200 batched B+tree (Python front end over the C ABI).

The compute path is libeirene_b200.so (hand-written sm_100a kernels behind the
C ABI in include/eirene_b200.h).  This module only loads the library and
passes device pointers (torch CUDA tensors) or host arrays through ctypes; it
has no fallback: if the library or a GPU is missing, calls raise.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libeirene_b200.so")

BT_OK = 0
ERRORS = {
    -1: "invalid argument",
    -2: "CUDA error",
    -3: "out of memory",
    -4: "node pool exhausted",
    -5: "reserved key UINT64_MAX",
    -6: "batch larger than max_batch",
    -7: "learned predictor not trained",
    -8: "more keys than BT_STATIC_BUILD_MAX_KEYS",
    -9: "no free slot or arena space",
    -10: "timed out",
    -11: "snapshot file error",
}
STATIC_BUILD_MAX_KEYS = 65536
OP_INSERT, OP_GET, OP_DELETE = 0, 1, 2
ST_ABSENT, ST_FOUND, ST_REJECTED, ST_RETRY_EXHAUSTED, ST_NO_CAPACITY = 0, 1, 2, 3, 4
MODE_SORTED, MODE_STM, MODE_MERGE_ENGINE = 0, 1, 0x10
DESCENT_PLAIN, DESCENT_LEARNED = 0, 1
DIST = {"uniform": 0, "zipf": 1, "normal": 2, "gamma": 3}
KEY_MAX = (1 << 64) - 1


class BTError(RuntimeError):
    def __init__(self, code: int, what: str = ""):
        super().__init__(f"{what}: {ERRORS.get(code, code)} ({code})")
        self.code = code


class Config(ctypes.Structure):
    _fields_ = [
        ("max_keys", ctypes.c_uint64),
        ("max_batch", ctypes.c_uint64),
        ("leaf_fill", ctypes.c_uint32),
        ("inner_fill", ctypes.c_uint32),
        ("retry_limit", ctypes.c_uint32),
        ("device", ctypes.c_int32),
        ("search_group", ctypes.c_uint32),
        ("n_segments", ctypes.c_uint32),
        ("window", ctypes.c_uint32),
        ("reserved", ctypes.c_uint32 * 7),
    ]


class Stats(ctypes.Structure):
    _fields_ = [
        ("n_keys", ctypes.c_uint64),
        ("n_nodes", ctypes.c_uint64),
        ("n_leaves", ctypes.c_uint64),
        ("height", ctypes.c_uint32),
        ("error", ctypes.c_uint32),
        ("commits", ctypes.c_uint64),
        ("aborts", ctypes.c_uint64),
        ("leaf_splits", ctypes.c_uint64),
        ("inner_splits", ctypes.c_uint64),
        ("new_roots", ctypes.c_uint64),
        ("retry_exhausted", ctypes.c_uint64),
        ("learned_hits", ctypes.c_uint64),
        ("learned_fallbacks", ctypes.c_uint64),
        ("learned_probe_sum", ctypes.c_uint64),
        ("capacity_nodes", ctypes.c_uint64),
    ]


class ServeConfig(ctypes.Structure):
    _fields_ = [("arena_bytes", ctypes.c_uint64), ("max_batches", ctypes.c_uint32), ("idle_us", ctypes.c_uint32),
                ("policy", ctypes.c_uint32), ("reserved", ctypes.c_uint32 * 5)]


class ServeStats(ctypes.Structure):
    _fields_ = [("batches", ctypes.c_uint64), ("requests", ctypes.c_uint64), ("kernel_launches", ctypes.c_uint64),
                ("in_flight", ctypes.c_uint64), ("p50_ms", ctypes.c_double), ("p99_ms", ctypes.c_double),
                ("max_ms", ctypes.c_double), ("mean_ms", ctypes.c_double), ("mops", ctypes.c_double),
                ("p50_service_ms", ctypes.c_double), ("p99_service_ms", ctypes.c_double),
                ("device_mops", ctypes.c_double)]


# every symbol the C header declares (checked by the CPU tests)
EXPORTS = [
    "bt_config_init", "bt_create", "bt_destroy", "bt_bulk_build", "bt_execute_batch", "bt_execute_batch_host",
    "bt_search_batch", "bt_insert_batch", "bt_size", "bt_dump_sorted", "bt_leaf_sizes", "bt_level_counts",
    "bt_stats_get", "bt_stats_reset", "bt_retrain", "bt_set_descent", "bt_set_root_model", "bt_set_search_group",
    "bt_host_alloc", "bt_host_free", "bt_gen_keys", "bt_gen_requests", "bt_status_string",
    "bt_profile", "bt_profile_read", "bt_launch_count", "bt_bulk_build_static",
    "bt_set_learned_group", "bt_learned_info", "bt_mlp_grad", "bt_set_option", "bt_autotune",
    "bt_serve_config_init", "bt_serve_start", "bt_submit", "bt_poll", "bt_wait", "bt_serve_get_stats", "bt_serve_stop",
    "bt_route_batch", "bt_unroute_results", "bt_save", "bt_load", "bt_range_batch", "bt_sync", "bt_save_image", "bt_load_image",
    "bt_refit", "bt_execute_batch_host_async", "bt_host_wait", "bt_serve_batch_times", "bt_autotune_fill",
    "bt_execute_batch_host_packed_async", "bt_execute_batches",
]
MAX_SHARDS = 256
OPT_SORTED_SEARCH, OPT_RETRY_LIMIT, OPT_TRAIN_STEPS, OPT_SORTED_LEAF_VALS, OPT_BATCH_DESCENT = 1, 2, 3, 4, 5
OPT_FRONT_END, OPT_TOP_CACHE, OPT_SEARCH_PAIRS, OPT_OVERLAP, OPT_ASYNC_WRITE = 6, 7, 8, 9, 10
OPT_REFIT_STEPS, OPT_LEARNED_MODE, OPT_HOST_VALUES_IN_PLACE, OPT_SORT_TILE, OPT_STM_COMBINE = 11, 12, 13, 14, 15
OPT_LEARNED_POLICY, OPT_HOST_FRONT_OVERLAP, OPT_TOUCH_SORT = 16, 17, 18
PHASES = ["sort", "merge", "search", "insert", "writeback"]

_lib = None
_P = ctypes.c_void_p
_SZ = ctypes.c_size_t


def build(force: bool = False) -> str:
    """Compile libeirene_b200.so in place (nvcc, sm_100a)."""
    import importlib

    mod = importlib.import_module(__name__ + ".build")
    # importing the submodule binds it as this package's `build` attribute:
    # put the function back so that later calls still reach it
    globals()["build"] = _build_fn
    return mod.build(force=force)


_build_fn = build


def lib():
    """Load libeirene_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: run `python -m eirene_b200.build` (needs nvcc)")
        L = ctypes.CDLL(LIB_PATH)
        sig = {
            "bt_config_init": [ctypes.POINTER(Config)],
            "bt_create": [ctypes.POINTER(Config), ctypes.POINTER(_P)],
            "bt_destroy": [_P],
            "bt_bulk_build": [_P, _P, _P, _SZ, _P],
            "bt_execute_batch": [_P, _P, _P, _P, _P, _P, _SZ, ctypes.c_int, _P],
            "bt_execute_batch_host": [_P, _P, _P, _P, _P, _P, _SZ, ctypes.c_int, _P],
            "bt_search_batch": [_P, _P, _P, _P, _SZ, _P],
            "bt_insert_batch": [_P, _P, _P, _P, _P, _SZ, _P],
            "bt_size": [_P, ctypes.POINTER(ctypes.c_uint64)],
            "bt_dump_sorted": [_P, _P, _P, _SZ, ctypes.POINTER(_SZ), _P],
            "bt_leaf_sizes": [_P, _P, _SZ, ctypes.POINTER(_SZ)],
            "bt_level_counts": [_P, _P, ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint32)],
            "bt_stats_get": [_P, ctypes.POINTER(Stats), ctypes.c_int],
            "bt_stats_reset": [_P],
            "bt_retrain": [_P, _P],
            "bt_refit": [_P, _P],
            "bt_execute_batch_host_async": [_P, _P, _P, _P, _P, _P, _SZ, ctypes.c_int, _P,
                                            ctypes.POINTER(ctypes.c_uint64)],
            "bt_execute_batch_host_packed_async": [_P, _P, _P, _P, _SZ, _P, _P, _SZ, ctypes.c_int, _P,
                                                   ctypes.POINTER(ctypes.c_uint64)],
            "bt_execute_batches": [_P, _SZ, _P, _P, _P, _P, _P, _P, ctypes.c_int, _P],
            "bt_host_wait": [_P, ctypes.c_uint64],
            "bt_serve_batch_times": [_P, ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64),
                                     ctypes.POINTER(ctypes.c_uint64)],
            "bt_set_descent": [_P, ctypes.c_int],
            "bt_set_root_model": [_P, ctypes.c_int],
            "bt_set_search_group": [_P, ctypes.c_uint32],
            "bt_host_alloc": [ctypes.POINTER(_P), _SZ],
            "bt_host_free": [_P],
            "bt_gen_keys": [ctypes.c_int, ctypes.c_uint64, _SZ, _P, _P, _P],
            "bt_gen_requests": [ctypes.c_int, ctypes.c_uint64, _P, _SZ, _SZ, ctypes.c_uint32, _P, _P, _P, _P],
            "bt_status_string": [ctypes.c_int],
            "bt_profile": [_P, ctypes.c_int],
            "bt_profile_read": [_P, _P, ctypes.POINTER(ctypes.c_uint64), ctypes.c_int],
            "bt_launch_count": [],
            "bt_bulk_build_static": [_P, _P, _P, _SZ, _P],
            "bt_set_learned_group": [_P, ctypes.c_uint32],
            "bt_learned_info": [_P, _P],
            "bt_mlp_grad": [_P, _P, _P, _P, _SZ, _P, _P, _P],
            "bt_set_option": [_P, ctypes.c_int, ctypes.c_int64],
            "bt_autotune": [_P, _P, _SZ, _P, _P],
            "bt_autotune_fill": [_P, _P, _SZ, _P, _P],
            "bt_serve_config_init": [ctypes.POINTER(ServeConfig)],
            "bt_serve_start": [_P, ctypes.POINTER(ServeConfig), ctypes.POINTER(_P)],
            "bt_submit": [_P, _P, _P, _P, _SZ, _P, _P, ctypes.POINTER(ctypes.c_uint64)],
            "bt_poll": [_P, ctypes.c_uint64, ctypes.POINTER(ctypes.c_int)],
            "bt_wait": [_P, ctypes.c_uint64, ctypes.c_uint32],
            "bt_serve_get_stats": [_P, ctypes.POINTER(ServeStats), ctypes.c_int],
            "bt_serve_stop": [_P],
            "bt_route_batch": [_P, _P, ctypes.c_int, _P, _P, _P, _SZ, _P, _P, _P, _P, _P, _P],
            "bt_unroute_results": [_P, _P, _P, _P, _SZ, _P, _P, _P],
            "bt_save": [_P, ctypes.c_char_p],
            "bt_range_batch": [_P, _P, _P, _SZ, ctypes.c_uint32, _P, _P, _P, _P],
            "bt_sync": [_P, _P],
            "bt_save_image": [_P, ctypes.c_char_p],
            "bt_load_image": [_P, ctypes.c_char_p],
            "bt_load": [_P, ctypes.c_char_p],
        }
        for name, args in sig.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = ctypes.c_int
        L.bt_status_string.restype = ctypes.c_char_p
        L.bt_launch_count.restype = ctypes.c_uint64
        _lib = L
    return _lib


def _check(rc: int, what: str):
    if rc != BT_OK:
        raise BTError(rc, what)


def _ptr(t) -> int:
    """Device pointer of a torch tensor (or an int already)."""
    if t is None:
        return None
    if isinstance(t, int):
        return t
    return t.data_ptr()


def _stream_ptr(stream) -> int | None:
    if stream is None:
        return None
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


class BTree:
    """One device-resident B+tree (one bt_handle)."""

    def __init__(self, max_keys: int = 1 << 20, max_batch: int = 1 << 22, leaf_fill: int = 24,
                 inner_fill: int = 24, device: int = 0, search_group: int = 4, retry_limit: int = 0,
                 n_segments: int = 0, window: int = 64):
        L = lib()
        cfg = Config()
        _check(L.bt_config_init(ctypes.byref(cfg)), "bt_config_init")
        cfg.max_keys = max_keys
        cfg.max_batch = max_batch
        cfg.leaf_fill = leaf_fill
        cfg.inner_fill = inner_fill
        cfg.device = device
        cfg.search_group = search_group
        if retry_limit:
            cfg.retry_limit = retry_limit
        cfg.n_segments = n_segments
        cfg.window = window
        h = _P()
        _check(L.bt_create(ctypes.byref(cfg), ctypes.byref(h)), "bt_create")
        self._h = h
        self.device = device
        self.max_batch = max_batch

    def close(self):
        if getattr(self, "_h", None):
            lib().bt_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # --- device-pointer API (torch CUDA tensors of dtype uint64 / uint8) ---
    def bulk_build(self, keys, vals, stream=None):
        n = keys.numel()
        _check(lib().bt_bulk_build(self._h, _ptr(keys), _ptr(vals), n, _stream_ptr(stream)), "bt_bulk_build")

    def execute(self, keys, vals, ops, out_vals, out_status, mode=MODE_SORTED, stream=None):
        n = keys.numel()
        _check(lib().bt_execute_batch(self._h, _ptr(keys), _ptr(vals), _ptr(ops), _ptr(out_vals), _ptr(out_status),
                                      n, mode, _stream_ptr(stream)), "bt_execute_batch")

    def search(self, keys, out_vals, out_status, stream=None):
        _check(lib().bt_search_batch(self._h, _ptr(keys), _ptr(out_vals), _ptr(out_status), keys.numel(),
                                     _stream_ptr(stream)), "bt_search_batch")

    def insert(self, keys, vals, out_vals, out_status, stream=None):
        _check(lib().bt_insert_batch(self._h, _ptr(keys), _ptr(vals), _ptr(out_vals), _ptr(out_status),
                                     keys.numel(), _stream_ptr(stream)), "bt_insert_batch")

    # --- host-buffer API (numpy arrays) ---
    def execute_host(self, keys: np.ndarray, vals: np.ndarray, ops: np.ndarray, mode=MODE_SORTED, stream=None,
                     out_vals: np.ndarray | None = None, out_status: np.ndarray | None = None):
        keys = np.ascontiguousarray(keys, dtype=np.uint64)
        vals = np.ascontiguousarray(vals, dtype=np.uint64)
        ops = np.ascontiguousarray(ops, dtype=np.uint8)
        n = keys.size
        if out_vals is None:
            out_vals = np.zeros(n, np.uint64)
        if out_status is None:
            out_status = np.zeros(n, np.uint8)
        _check(lib().bt_execute_batch_host(self._h, keys.ctypes.data, vals.ctypes.data, ops.ctypes.data,
                                           out_vals.ctypes.data, out_status.ctypes.data, n, mode,
                                           _stream_ptr(stream)), "bt_execute_batch_host")
        return out_vals, out_status

    def submit_host(self, keys, vals, ops, out_vals, out_status, mode=MODE_SORTED, stream=None) -> int:
        """bt_execute_batch_host_async over host buffers (numpy arrays or CPU
        tensors, kept alive and unchanged by the caller until wait_host);
        returns the ticket."""
        def addr(a):
            return a.data_ptr() if hasattr(a, "data_ptr") else a.ctypes.data

        n = keys.numel() if hasattr(keys, "numel") else keys.size
        t = ctypes.c_uint64(0)
        _check(lib().bt_execute_batch_host_async(self._h, addr(keys), addr(vals), addr(ops), addr(out_vals),
                                                 addr(out_status), n, mode, _stream_ptr(stream), ctypes.byref(t)),
               "bt_execute_batch_host_async")
        return t.value

    def submit_host_packed(self, keys, ops, insert_vals, out_vals, out_status, mode=MODE_SORTED,
                           stream=None) -> int:
        """bt_execute_batch_host_packed_async: like submit_host, with the values
        of the batch's INSERTs only (insert_vals[j] belongs to the j-th INSERT
        in request order); returns the ticket."""
        def addr(a):
            return a.data_ptr() if hasattr(a, "data_ptr") else a.ctypes.data

        n = keys.numel() if hasattr(keys, "numel") else keys.size
        m = insert_vals.numel() if hasattr(insert_vals, "numel") else insert_vals.size
        t = ctypes.c_uint64(0)
        _check(lib().bt_execute_batch_host_packed_async(self._h, addr(keys), addr(ops), addr(insert_vals) if m else None,
                                                        m, addr(out_vals), addr(out_status), n, mode,
                                                        _stream_ptr(stream), ctypes.byref(t)),
               "bt_execute_batch_host_packed_async")
        return t.value

    def execute_many(self, batches, outs, mode=MODE_SORTED, stream=None):
        """bt_execute_batches: `batches` a list of (keys, vals, ops) CUDA
        tensors, `outs` a list of (out_vals, out_status), one per batch."""
        m = len(batches)
        if len(outs) != m:
            raise ValueError("one (out_vals, out_status) per batch")
        arr = lambda xs: (ctypes.c_void_p * max(m, 1))(*[_ptr(x) for x in xs])
        ns = (_SZ * max(m, 1))(*[b[0].numel() for b in batches])
        _check(lib().bt_execute_batches(self._h, m, arr([b[0] for b in batches]), arr([b[1] for b in batches]),
                                        arr([b[2] for b in batches]), arr([o[0] for o in outs]),
                                        arr([o[1] for o in outs]), ns, mode, _stream_ptr(stream)),
               "bt_execute_batches")

    def wait_host(self, ticket: int):
        _check(lib().bt_host_wait(self._h, ticket), "bt_host_wait")

    def size(self) -> int:
        v = ctypes.c_uint64(0)
        _check(lib().bt_size(self._h, ctypes.byref(v)), "bt_size")
        return v.value

    def dump(self):
        """Sorted (keys, vals) as int64 torch CUDA tensors holding the uint64 bit patterns."""
        import torch

        n = self.size()
        k = torch.empty(max(n, 1), dtype=torch.int64, device=f"cuda:{self.device}")
        v = torch.empty(max(n, 1), dtype=torch.int64, device=f"cuda:{self.device}")
        got = _SZ(0)
        _check(lib().bt_dump_sorted(self._h, _ptr(k), _ptr(v), k.numel(), ctypes.byref(got), None), "bt_dump_sorted")
        return k[: got.value], v[: got.value]

    def leaf_sizes(self) -> np.ndarray:
        n = _SZ(0)
        _check(lib().bt_leaf_sizes(self._h, None, 0, ctypes.byref(n)), "bt_leaf_sizes")
        out = np.zeros(n.value, np.uint32)
        if n.value:
            _check(lib().bt_leaf_sizes(self._h, out.ctypes.data, n.value, ctypes.byref(n)), "bt_leaf_sizes")
        return out

    def level_counts(self) -> np.ndarray:
        c = np.zeros(48, np.uint64)
        h = ctypes.c_uint32(0)
        _check(lib().bt_level_counts(self._h, c.ctypes.data, 48, ctypes.byref(h)), "bt_level_counts")
        return c[: h.value]

    def stats(self, with_leaves: bool = False) -> dict:
        s = Stats()
        _check(lib().bt_stats_get(self._h, ctypes.byref(s), 1 if with_leaves else 0), "bt_stats_get")
        return {f: getattr(s, f) for f, _ in Stats._fields_}

    def reset_stats(self):
        _check(lib().bt_stats_reset(self._h), "bt_stats_reset")

    def retrain(self, stream=None):
        _check(lib().bt_retrain(self._h, _stream_ptr(stream)), "bt_retrain")

    def refit(self, stream=None):
        """Incremental retraining: the leaf array and segment lines follow the
        current leaves; the trained stage-1 model is kept."""
        _check(lib().bt_refit(self._h, _stream_ptr(stream)), "bt_refit")

    def set_descent(self, learned: bool):
        _check(lib().bt_set_descent(self._h, DESCENT_LEARNED if learned else DESCENT_PLAIN), "bt_set_descent")

    def set_root_model(self, mlp: bool):
        _check(lib().bt_set_root_model(self._h, 1 if mlp else 0), "bt_set_root_model")

    def profile(self, enable: bool = True):
        _check(lib().bt_profile(self._h, 1 if enable else 0), "bt_profile")

    def profile_read(self, reset: bool = True) -> dict:
        ms = (ctypes.c_double * 5)()
        b = ctypes.c_uint64(0)
        _check(lib().bt_profile_read(self._h, ms, ctypes.byref(b), 1 if reset else 0), "bt_profile_read")
        return {"batches": b.value, **{p: ms[i] for i, p in enumerate(PHASES)}}

    def sync(self, stream=None):
        """Order `stream` (or, with None, the host) after every batch issued so
        far, the deferred leaf/inner merge included (OPT_ASYNC_WRITE)."""
        _check(lib().bt_sync(self._h, _stream_ptr(stream)), "bt_sync")

    def set_option(self, option: int, value: int):
        _check(lib().bt_set_option(self._h, option, value), "bt_set_option")

    def autotune(self, sample_keys, stream=None) -> dict:
        rep = (ctypes.c_double * 24)()
        _check(lib().bt_autotune(self._h, _ptr(sample_keys), sample_keys.numel(), _stream_ptr(stream), rep),
               "bt_autotune")
        r = list(rep)
        return {"plain_lanes": int(r[0]), "learned_lanes": int(r[1]), "sorted_leaf_vals": int(r[2]),
                "batch_descent": "learned" if r[3] == 1 else "plain",
                "learned_mode": int(r[15]),
                "plain_ms": dict(zip([4, 8, 16, 32], r[4:8])),
                "learned_ms": dict(zip(["4 pipelined", "2 pipelined", "4x1", "2x1"], r[8:12])),
                "sorted_plain_ms": r[12:14], "sorted_learned_ms": r[14],
                "sort_threads": int(r[16]), "sort_threads_touched": int(r[17]),
                "sort_ms": dict(zip([256, 512, 1024], r[18:21])),
                "sort_touched_ms": dict(zip([256, 512, 1024], r[21:24]))}

    def autotune_fill(self, sample_keys, stream=None) -> dict:
        """bt_autotune_fill: the node fill for later bulk builds and splits,
        chosen by timing batches on sample trees."""
        rep = (ctypes.c_double * 8)()
        _check(lib().bt_autotune_fill(self._h, _ptr(sample_keys), sample_keys.numel(), _stream_ptr(stream), rep),
               "bt_autotune_fill")
        r = list(rep)
        return {"leaf_fill": int(r[0]), "inner_fill": int(r[1]), "batch_ms": dict(zip([16, 20, 24, 28], r[2:6]))}

    def set_learned_group(self, lanes: int):
        _check(lib().bt_set_learned_group(self._h, lanes), "bt_set_learned_group")

    def learned_info(self) -> dict:
        a = (ctypes.c_double * 8)()
        _check(lib().bt_learned_info(self._h, a), "bt_learned_info")
        keys = ["valid", "n_leaves", "n_segments", "segments_over_window", "window", "loss", "root_mlp", "steps"]
        return {k: a[i] for i, k in enumerate(keys)}

    def mlp_grad(self, params, x, y, grad_out, loss_out, stream=None):
        _check(lib().bt_mlp_grad(self._h, _ptr(params), _ptr(x), _ptr(y), x.numel(), _ptr(grad_out),
                                 _ptr(loss_out), _stream_ptr(stream)), "bt_mlp_grad")

    def route(self, splitters, n_shards: int, keys, vals, ops, out_keys, out_vals, out_ops, out_perm, out_counts,
              stream=None):
        """Stable partition of a batch by owning shard (bt_route_batch)."""
        _check(lib().bt_route_batch(self._h, _ptr(splitters), n_shards, _ptr(keys), _ptr(vals), _ptr(ops), keys.numel(),
                                    _ptr(out_keys), _ptr(out_vals), _ptr(out_ops), _ptr(out_perm), _ptr(out_counts),
                                    _stream_ptr(stream)), "bt_route_batch")

    def unroute(self, perm, in_vals, in_status, out_vals, out_status, stream=None):
        """Scatter answers in routed order back to input order (bt_unroute_results)."""
        _check(lib().bt_unroute_results(self._h, _ptr(perm), _ptr(in_vals), _ptr(in_status), perm.numel(),
                                        _ptr(out_vals), _ptr(out_status), _stream_ptr(stream)), "bt_unroute_results")

    def range(self, lo, hi, max_per: int, stream=None):
        """Range scan of [lo[i], hi[i]] (int64 CUDA tensors of uint64 bit patterns):
        (counts int32 [n], keys [n, max_per], vals [n, max_per]); counts above
        max_per mean the query was truncated."""
        import torch

        n = lo.numel()
        dev_ = lo.device
        keys = torch.zeros((n, max(max_per, 1)), dtype=torch.int64, device=dev_)[:, :max_per]
        vals = torch.zeros((n, max(max_per, 1)), dtype=torch.int64, device=dev_)[:, :max_per]
        counts = torch.zeros(max(n, 1), dtype=torch.int32, device=dev_)[:n]
        _check(lib().bt_range_batch(self._h, _ptr(lo), _ptr(hi), n, max_per, _ptr(keys), _ptr(vals), _ptr(counts),
                                    _stream_ptr(stream)), "bt_range_batch")
        return counts, keys, vals

    def save(self, path: str):
        """Write the tree's sorted pairs to a snapshot file (bt_save)."""
        _check(lib().bt_save(self._h, os.fsencode(path)), "bt_save")

    def load(self, path: str):
        """Replace the contents with a snapshot file (bt_load; a fresh bulk load)."""
        _check(lib().bt_load(self._h, os.fsencode(path)), "bt_load")

    def save_image(self, path: str):
        """Write the node pool itself to a file (bt_save_image)."""
        _check(lib().bt_save_image(self._h, os.fsencode(path)), "bt_save_image")

    def load_image(self, path: str):
        """Restore a pool image, leaf layout included (bt_load_image)."""
        _check(lib().bt_load_image(self._h, os.fsencode(path)), "bt_load_image")

    def set_search_group(self, lanes: int):
        _check(lib().bt_set_search_group(self._h, lanes), "bt_set_search_group")


class HostBuffer:
    """Page-locked host memory from bt_host_alloc for the host-buffer entry
    point (copies to and from it run at the link's full speed without a
    staging copy); `tensor` is a CPU tensor over it.  free() releases it:
    the tensor must not be used after that."""

    def __init__(self, n: int, dtype):
        import torch

        nbytes = max(1, n * torch.empty(0, dtype=dtype).element_size())
        p = _P()
        _check(lib().bt_host_alloc(ctypes.byref(p), nbytes), "bt_host_alloc")
        self._p = p.value
        buf = (ctypes.c_uint8 * nbytes).from_address(self._p)
        self.tensor = torch.from_numpy(np.ctypeslib.as_array(buf)).view(dtype)[:n]

    def free(self):
        if self._p:
            self.tensor = None
            _check(lib().bt_host_free(self._p), "bt_host_free")
            self._p = None


def launch_count() -> int:
    return lib().bt_launch_count()


def gen_keys(dist: str, seed: int, n: int, keys, vals=None, stream=None):
    _check(lib().bt_gen_keys(DIST[dist], seed, n, _ptr(keys), _ptr(vals), _stream_ptr(stream)), "bt_gen_keys")


def gen_requests(dist: str, seed: int, tree_keys, n: int, search_pct: int, keys, vals, ops, stream=None):
    nt = 0 if tree_keys is None else tree_keys.numel()
    _check(lib().bt_gen_requests(DIST[dist], seed, _ptr(tree_keys), nt, n, search_pct, _ptr(keys), _ptr(vals),
                                 _ptr(ops), _stream_ptr(stream)), "bt_gen_requests")


class Server:
    """Continuous-batching server over one BTree (host numpy buffers)."""

    def __init__(self, tree: "BTree", arena_bytes: int = 1 << 30, max_batches: int = 256, idle_us: int = 2000,
                 policy: int = 0):
        cfg = ServeConfig()
        _check(lib().bt_serve_config_init(ctypes.byref(cfg)), "bt_serve_config_init")
        cfg.arena_bytes, cfg.max_batches, cfg.idle_us, cfg.policy = arena_bytes, max_batches, idle_us, policy
        h = _P()
        _check(lib().bt_serve_start(tree._h, ctypes.byref(cfg), ctypes.byref(h)), "bt_serve_start")
        self._s = h
        self.tree = tree
        self._keep = {}

    def submit(self, keys, vals, ops, out_vals, out_status):
        """Returns a ticket, or None when the server is busy (no slot / arena space)."""
        t = ctypes.c_uint64(0)
        rc = lib().bt_submit(self._s, keys.ctypes.data, vals.ctypes.data, ops.ctypes.data, keys.size,
                             out_vals.ctypes.data, out_status.ctypes.data, ctypes.byref(t))
        if rc == -9:
            return None
        _check(rc, "bt_submit")
        self._keep[t.value] = (keys, vals, ops, out_vals, out_status)
        return t.value

    def poll(self, ticket) -> bool:
        d = ctypes.c_int(0)
        _check(lib().bt_poll(self._s, ticket, ctypes.byref(d)), "bt_poll")
        if d.value == 1:
            self._keep.pop(ticket, None)
        return d.value == 1

    def wait(self, ticket, timeout_ms: int = 120000):
        _check(lib().bt_wait(self._s, ticket, timeout_ms), "bt_wait")
        self._keep.pop(ticket, None)

    def batch_times(self, ticket) -> tuple[int, int]:
        """(first claimed chunk, completion) of a finished batch, device clock in ns."""
        a, b = ctypes.c_uint64(0), ctypes.c_uint64(0)
        _check(lib().bt_serve_batch_times(self._s, ticket, ctypes.byref(a), ctypes.byref(b)), "bt_serve_batch_times")
        return a.value, b.value

    def stats(self, reset: bool = False) -> dict:
        st = ServeStats()
        _check(lib().bt_serve_get_stats(self._s, ctypes.byref(st), 1 if reset else 0), "bt_serve_get_stats")
        return {f: getattr(st, f) for f, _ in ServeStats._fields_}

    def stop(self):
        if getattr(self, "_s", None):
            lib().bt_serve_stop(self._s)
            self._s = None
            self._keep.clear()

    def __del__(self):
        try:
            self.stop()
        except Exception:
            pass
