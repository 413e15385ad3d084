#!/usr/bin/env python
"""Throughput of the batched B+tree on B200: Mops/s at 2^26 uint64 keys with a
95% search / 5% insert mix, batches of 2^22 requests through the sort-based
batch merge (the reference's v38 meaning), plain and learned descent, p50/p99
batch latency.

One step = one bt_execute_batch over a fresh, device-resident batch of 2^22
seeded synthetic requests (the reference's dataset files are not shipped; the
generator reproduces their shape: 95% reads, half of them existing keys).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun the ranks hold one key-range-sharded tree (eirene_b200.shard):
each rank builds from its own 2^26 keys, the splitters are quantiles of all
ranks' keys, and every step each rank submits its own 2^22-request batch,
which is routed to the owning GPUs by an all-to-all over NCCL, run there, and
answered by the reverse all-to-all (weak scaling: keys and requests per GPU are
fixed).  Rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import ctypes
import datetime
import json
import os
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mops/s at 2^26 keys, 95% search; learned vs plain descent; p99 batch latency"
BYTES_SEARCH = 288  # leaf keys (256 B) + one 32 B value sector
BYTES_INSERT = 864  # search bytes + leaf rewrite (512 B) + version acquire/release (64 B)
BYTES_SORT = 192  # 8 radix passes x (8 B key + 4 B index) x (read + write)
FALLBACK_HBM_GBS = 6650.0


def env_int(name, default):
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """SM clock and throttle-reason samples taken while the timed region runs.

    Reads NVML (nvidia-ml-py) every 2 ms from a host thread (the timed region
    is tens of milliseconds, too short for nvidia-smi's sampling interval);
    falls back to `nvidia-smi -lms 200` where NVML is not importable.  Only
    reads: it changes no setting of the GPU."""

    NVML_REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
                    ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
                    ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
                    ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"),
                    ("hw_power_brake_slowdown", "nvmlClocksEventReasonHwPowerBrakeSlowdown"))
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, cuda_index: int):
        self.cuda_index = cuda_index
        self.proc = None
        self.thread = None
        self.samples = []
        self.reasons = set()
        self.max_mhz = 0.0
        self.source = None

    def start(self):
        import threading

        try:
            import pynvml
            import torch

            pynvml.nvmlInit()
            try:
                idx = torch.cuda._get_nvml_device_index(self.cuda_index)
            except Exception:
                idx = self.cuda_index
            h = pynvml.nvmlDeviceGetHandleByIndex(idx)
            self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))
            bits = [(nm, getattr(pynvml, c)) for nm, c in self.NVML_REASONS if hasattr(pynvml, c)]
            self.stop_flag = threading.Event()

            def run():
                while not self.stop_flag.is_set():
                    try:
                        self.samples.append(float(pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)))
                        r = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
                        for nm, b in bits:
                            if r & b:
                                self.reasons.add(nm)
                    except Exception:
                        pass
                    self.stop_flag.wait(0.002)

            self.thread = threading.Thread(target=run, daemon=True)
            self.thread.start()
            self.source = "nvml, 2 ms"
            return
        except Exception:
            self.thread = None
        try:
            self.path = os.path.join("/tmp", f"bt_clocks_{os.getpid()}.csv")
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.cuda_index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.fh, stderr=subprocess.DEVNULL)
            self.source = "nvidia-smi, 200 ms"
        except Exception:
            self.proc = None

    def stop(self):
        if self.thread is not None:
            self.stop_flag.set()
            self.thread.join(2)
            try:
                import pynvml

                pynvml.nvmlShutdown()
            except Exception:
                pass
        elif self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.fh.close()
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) < 9:
                    continue
                try:
                    self.samples.append(float(f[1]))
                    self.max_mhz = max(self.max_mhz, float(f[2]))
                except ValueError:
                    continue
                for nm, v in zip(names, f[5:9]):
                    if v.lower().startswith("active"):
                        self.reasons.add(nm)
        if not self.samples:
            return None
        sm = sorted(self.samples)
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons),
                "samples": len(sm), "source": self.source}


# ----------------------------------------------------------------------------
# The reference program's own benchmark shape, for a same-box comparison with
# its GPU build: a tree built from 2^23 - 1 `P` lines, then query files of 95 %
# `R` / 5 % `P` lines (half the reads hit tree keys), run in batches of
# 1,310,720 (evalutaion/random_testall_v39.sh:9-28, prof/query23_uniform_95_v39.res,
# src/gpu-stm-tree-v39/bpt-gpustm.h:25-38).  Keys are 31-bit: the reference
# is int32 with INT_MAX reserved.  The reference arm runs the reference
# program on these inputs; this library's arm runs itself on the same ones.
REF_BATCH = 1_310_720


def _mix64(x):
    import numpy as np

    x = x.astype(np.uint64)
    with np.errstate(over="ignore"):
        x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return x ^ (x >> np.uint64(31))


def _key31(seed: int, n: int):
    """n distinct keys in [0, 2^31 - 1), in a seeded random order."""
    import numpy as np

    out = np.zeros(0, np.uint64)
    c = 0
    while out.size < n:
        i = np.arange(c, c + 2 * n, dtype=np.uint64)
        with np.errstate(over="ignore"):
            k = _mix64(i * np.uint64(0x9E3779B97F4A7C15) + np.uint64(seed)) >> np.uint64(33)
        out = np.unique(np.concatenate([out, k[k < np.uint64(2**31 - 1)]]))
        c += 2 * n
    return np.random.default_rng(seed).permutation(out)[:n]


def ref31_workload(batches: int = 10, tree: int = (1 << 23) - 1):
    """(build keys, build values, query keys, query values, query op codes)."""
    import numpy as np

    pool = _key31(77, tree + batches * REF_BATCH)
    bk, fresh = pool[:tree], pool[tree:]
    bv = (bk * np.uint64(7) + np.uint64(3)) & np.uint64(0x7FFFFFFF)
    rng = np.random.default_rng(5)
    nq = batches * REF_BATCH
    is_get = rng.random(nq) < 0.95
    qk = np.where(rng.random(nq) < 0.5, bk[rng.integers(0, bk.size, nq)], fresh[rng.integers(0, fresh.size, nq)])
    qk = np.where(is_get, qk, fresh[rng.permutation(nq) % fresh.size])
    qo = np.where(is_get, 1, 0).astype(np.uint8)
    qv = (np.arange(nq, dtype=np.uint64) * np.uint64(13) + np.uint64(5)) & np.uint64(0x7FFFFFFF)
    return bk, bv, qk, qv, qo


def reference_gpu(ref_bin: str, batches: int = 10):
    """The reference program (built from its own sources into oracle/_ref) on
    the 31-bit workload: its "total gpu exec time" of the build file and of
    the query file (v39 times its kernel only, v38 all of its phases;
    src/gpu-stm-tree-v39/bpt-gpustm-kernel.cu:262-282,
    src/gpu-stm-tree-v38/bpt-gpustm-kernel.cu:289-324)."""
    import tempfile

    bk, bv, qk, qv, qo = ref31_workload(batches)
    out = {"tree_keys": int(bk.size), "requests": int(qk.size), "batch": REF_BATCH, "search_frac": 0.95}
    with tempfile.TemporaryDirectory() as d:
        b, q = os.path.join(d, "build.txt"), os.path.join(d, "query.txt")
        with open(b, "w") as f:
            f.write("".join(f"P {k} {v}\n" for k, v in zip(bk.tolist(), bv.tolist())))
        with open(q, "w") as f:
            f.write("".join(f"P {k} {v}\n" if o == 0 else f"R {k}\n"
                            for k, v, o in zip(qk.tolist(), qv.tolist(), qo.tolist())))
        for ver in (39, 38):
            t0 = time.time()
            try:
                r = subprocess.run([ref_bin, f"-v{ver}", "-i", b, "-i", q], capture_output=True, text=True,
                                   timeout=900)
            except subprocess.TimeoutExpired:
                out[f"v{ver}"] = {"error": "timeout"}
                continue
            times = [float(ln.split(":")[1]) for ln in r.stdout.splitlines() if "total gpu exec time" in ln]
            if r.returncode != 0 or len(times) < 2:
                out[f"v{ver}"] = {"error": (r.stdout + r.stderr)[-300:]}
                continue
            out[f"v{ver}"] = {"build_s": times[0], "query_s": times[1], "query_mops": qk.size / times[1] / 1e6,
                              "wall_s": time.time() - t0}
    return out


def stm_run(E, torch, t, keys_dev, n_b, warmup, steps, dist, search_pct, seed0, stream):
    """`warmup` then `steps` BT_MODE_STM batches of fresh requests drawn from
    `dist` over keys_dev; Mops/s over the timed batches and the STM counters."""
    bs = []
    for i in range(warmup + steps):
        k = torch.empty(n_b, dtype=torch.int64, device="cuda")
        v = torch.empty(n_b, dtype=torch.int64, device="cuda")
        o = torch.empty(n_b, dtype=torch.uint8, device="cuda")
        E.gen_requests(dist, seed0 + i, keys_dev, n_b, search_pct, k, v, o, stream)
        bs.append((k, v, o))
    ov = torch.empty(n_b, dtype=torch.int64, device="cuda")
    ost = torch.empty(n_b, dtype=torch.uint8, device="cuda")
    for i in range(warmup):
        t.execute(*bs[i], ov, ost, mode=E.MODE_STM, stream=stream)
    torch.cuda.synchronize()
    s0 = t.stats()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for i in range(warmup, warmup + steps):
        t.execute(*bs[i], ov, ost, mode=E.MODE_STM, stream=stream)
    e1.record(stream)
    torch.cuda.synchronize()
    s1 = t.stats()
    ms = e0.elapsed_time(e1)
    commits, aborts = s1["commits"] - s0["commits"], s1["aborts"] - s0["aborts"]
    return {"mops": n_b * steps / (ms / 1e3) / 1e6, "ms_per_batch": ms / steps, "commits": commits,
            "aborts": aborts, "aborts_per_commit": aborts / max(1, commits),
            "retry_exhausted": s1["retry_exhausted"] - s0["retry_exhausted"], "batches": steps}


def stm_passes(E, torch, tree, tk, n_b, steps, search_pct, stream):
    """BT_MODE_STM batches (the reference's v39 meaning: requests are
    concurrent warp transactions): on the headline tree with its workload, and
    on a skewed tree (Zipf(0.99) 2^25 keys, 95/5, the inserts drawn from the
    same Zipf law, so popular keys repeat and transactions collide).  Reports
    Mops/s and the STM counters: commits, aborts (the reference's
    ABORT_COUNT roll-backs, src/gpu-stm-tree-v39/bpt-gpustm-kernel.cu:58-63)
    and requests that exhausted the retry limit."""
    out = {}

    def run(t, keys_dev, dist, seed0):
        return stm_run(E, torch, t, keys_dev, n_b, 3, steps, dist, search_pct, seed0, stream)

    tree.set_descent(False)
    out["headline_tree"] = run(tree, tk, "uniform", 60_000)
    nz = 1 << 25
    zt = E.BTree(max_keys=2 * nz, max_batch=n_b)
    zk = torch.empty(nz, dtype=torch.int64, device="cuda")
    zv = torch.empty(nz, dtype=torch.int64, device="cuda")
    E.gen_keys("zipf", 2, nz, zk, zv, stream)
    zt.bulk_build(zk, zv, stream)
    del zv
    out["zipf_2e25"] = run(zt, zk, "zipf", 70_000)
    zt.close()
    del zk
    out["workload"] = (f"batches of {n_b} requests, {search_pct}% search, BT_MODE_STM; the headline tree, and a "
                       "Zipf(0.99) tree of 2^25 keys with Zipf-drawn (duplicate-heavy) inserts")
    return out


def same_box_ours(E, torch, batches: int = 10):
    """This library on the 31-bit workload the reference arm gives the
    reference program: the tree built by inserting the build file's pairs
    in batches of 1,310,720 (as the reference builds), then the query file
    in batches of 1,310,720, device-timed (CUDA events around the batches);
    the sorted batch meaning (the reference's v38) in both forms, and the
    STM meaning (v39)."""
    import numpy as np

    bk, bv, qk, qv, qo = ref31_workload(batches)
    k = torch.from_numpy(qk.view(np.int64)).cuda()
    v = torch.from_numpy(qv.view(np.int64)).cuda()
    o = torch.from_numpy(qo).cuda()
    bkt = torch.from_numpy(bk.view(np.int64)).cuda()
    bvt = torch.from_numpy(bv.view(np.int64)).cuda()
    bot = torch.zeros(bk.size, dtype=torch.uint8, device="cuda")
    ov = torch.empty(REF_BATCH, dtype=torch.int64, device="cuda")
    ost = torch.empty(REF_BATCH, dtype=torch.uint8, device="cuda")
    out = {"tree_keys": int(bk.size), "requests": int(qk.size), "batch": REF_BATCH, "search_frac": 0.95}
    MERGE = E.MODE_SORTED | E.MODE_MERGE_ENGINE
    for name, mode, learned in (("sorted_plain", MERGE, False), ("sorted_learned", MERGE, True),
                                ("stm", E.MODE_STM, False), ("stm_learned", E.MODE_STM, True)):
        t = E.BTree(max_keys=2 * bk.size + qk.size, max_batch=REF_BATCH)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for i in range(0, bk.size, REF_BATCH):
            s_ = slice(i, min(bk.size, i + REF_BATCH))
            t.execute(bkt[s_], bvt[s_], bot[s_], ov[: s_.stop - s_.start], ost[: s_.stop - s_.start], mode=MERGE)
        t.sync()
        e1.record()
        torch.cuda.synchronize()
        build_ms = e0.elapsed_time(e1)
        if learned:
            t.retrain()
            t.set_descent(True)
            t.autotune(k[:REF_BATCH])
        e0.record()
        for i in range(batches):
            s_ = slice(i * REF_BATCH, (i + 1) * REF_BATCH)
            t.execute(k[s_], v[s_], o[s_], ov, ost, mode=mode)
        t.sync()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        out[name] = {"build_s": build_ms / 1e3, "query_s": ms / 1e3, "query_mops": qk.size / (ms / 1e3) / 1e6}
        t.close()
    return out


def cpu_baseline(args, n_sample: int, threads: int):
    """The oracle (CPU restatement of the reference path; the reference has no
    CPU implementation) on a bounded sample of the same workload."""
    import numpy as np

    from oracle import oracle as O

    t0 = time.time()
    keys = O.gen_keys(args.dist, 1, 1 << args.tree_log2)
    tree = O.OracleTree(24, 24)
    tree.bulk_build(keys, O.value_of(keys))
    build_s = time.time() - t0
    rk, rv, ro = O.gen_requests(args.dist, 999, keys, n_sample, args.search_pct)
    t1 = time.perf_counter()
    tree.execute_merged(rk, rv, ro, O.ENGINE_STM, threads)
    dt = time.perf_counter() - t1
    # the same on one thread, on an eighth of the sample
    n1 = max(1, n_sample // 8)
    rk1, rv1, ro1 = O.gen_requests(args.dist, 998, keys, n1, args.search_pct)
    t1 = time.perf_counter()
    tree.execute_merged(rk1, rv1, ro1, O.ENGINE_STM, 1)
    dt1 = time.perf_counter() - t1
    del tree
    return {"value": n_sample / dt / 1e6, "unit": "Mops/s", "cores": threads, "kind": "port",
            "single_thread_value": n1 / dt1 / 1e6,
            "sample": f"{n_sample} requests ({args.search_pct}% search) of the bench workload against a "
                      f"2^{args.tree_log2}-key tree, sort-merged batch semantics; tree build ({build_s:.1f} s) untimed"}


def run_reference(args):
    """--impl reference: the reference's CPU implementation of the path does not
    exist (it is GPU-only), so the oracle port stands in for it, timed on the
    host cores with all threads."""
    rank = env_int("RANK", 0)
    if rank != 0:
        return 0
    import numpy as np

    from oracle import oracle as O

    threads = os.cpu_count() or 1
    keys = O.gen_keys(args.dist, 1, 1 << args.tree_log2)
    tree = O.OracleTree(24, 24)
    tree.bulk_build(keys, O.value_of(keys))
    n_step = 1 << 18
    batches = [O.gen_requests(args.dist, 5000 + i, keys, n_step, args.search_pct)
               for i in range(args.warmup + args.steps)]
    for i in range(args.warmup):
        tree.execute_merged(*batches[i], O.ENGINE_STM, threads)
    t0 = time.perf_counter()
    for i in range(args.warmup, args.warmup + args.steps):
        tree.execute_merged(*batches[i], O.ENGINE_STM, threads)
    dt = time.perf_counter() - t0
    val = n_step * args.steps / dt / 1e6
    line = {
        "impl": "reference", "metric": METRIC, "value": val, "unit": "Mops/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
        "config": {"workload": f"2^{args.tree_log2}-key tree, {args.search_pct}/{100 - args.search_pct} "
                               f"search/insert, {args.dist} keys, sort-merged batches",
                   "step_sample": n_step},
        "cpu_baseline": {"value": val, "unit": "Mops/s", "cores": threads, "kind": "port",
                         "sample": f"each step {n_step} requests of the bench workload (the reference has no "
                                   "CPU path; the oracle restatement runs in its place)"},
        "e2e": {"value": val, "unit": "Mops/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    # the reference's GPU build on this box, when it was compiled from the
    # reference's sources (oracle/_ref): its own benchmark shape, 31-bit keys
    ref_bin = os.path.join(ROOT, "oracle", "_ref", "stm_test")
    if not args.no_same_box:
        try:
            import torch

            has_gpu = torch.cuda.is_available()
        except Exception:
            has_gpu = False
        if not has_gpu:
            line["reference_gpu"] = {"unavailable": "no GPU on this machine"}
        elif os.path.exists(ref_bin):
            try:
                line["reference_gpu"] = reference_gpu(ref_bin)
            except Exception as ex:  # reported, not fatal
                line["reference_gpu"] = {"error": str(ex)}
        else:
            line["reference_gpu"] = {"unavailable": "oracle/_ref/stm_test was not built (no reference sources)"}
    print(json.dumps(line), flush=True)
    return 0


# ----------------------------------------------------------------------------
def serve_bench(E, np, tree, tk_host, n_tree, seconds=1.5, seed=5, load=0.5, policy=0, loads=(0.25, 0.5, 0.75)):
    """Serving loop (continuous batching): batch sizes log-uniform over
    2^10..2^22, per-batch search fraction uniform in [0.5, 1], Poisson arrivals.
    After a warm-up pass, phase 1 submits as fast as admission allows
    (saturated rate); then Poisson arrivals offer each fraction in `loads` of
    that rate, and each phase reports what was served, the batch latency and
    its device-side part (first claimed chunk to last finished one).  The
    sustainable rate is the highest offered one that was served in full
    (served >= 95 % of offered) with p99 <= 10 x p50."""
    import torch

    rng = np.random.default_rng(seed)
    n_pool = 1 << 22
    fracs = [0.5, 0.6, 0.7, 0.8, 0.9, 1.0]
    pools = []
    keep = []
    for i, f in enumerate(fracs):
        k = torch.empty(n_pool, dtype=torch.int64, device="cuda")
        v = torch.empty(n_pool, dtype=torch.int64, device="cuda")
        o = torch.empty(n_pool, dtype=torch.uint8, device="cuda")
        E.gen_requests("uniform", 50_000 + i, tk_host, n_pool, int(round(f * 100)), k, v, o)
        kp, vp, op = k.cpu().pin_memory(), v.cpu().pin_memory(), o.cpu().pin_memory()  # pinned host pools
        keep.append((kp, vp, op))
        pools.append((kp.numpy().view(np.uint64), vp.numpy().view(np.uint64), op.numpy()))
        del k, v, o
    ov_t = torch.empty(n_pool, dtype=torch.int64).pin_memory()
    os_t = torch.empty(n_pool, dtype=torch.uint8).pin_memory()
    out_v = ov_t.numpy().view(np.uint64)
    out_s = os_t.numpy()
    srv = E.Server(tree, arena_bytes=3 << 30, max_batches=512, policy=policy)

    def draw():
        n = int(2 ** rng.uniform(10, 22))
        p = pools[int(np.argmin([abs(f - rng.uniform(0.5, 1.0)) for f in fracs]))]
        off = int(rng.integers(0, n_pool - n + 1))
        return p[0][off:off + n], p[1][off:off + n], p[2][off:off + n], out_v[:n], out_s[:n]

    def run(duration, rate):
        srv.stats(reset=True)
        t0 = time.perf_counter()
        pending = []
        next_t = t0
        n_sub = 0
        busy = 0
        lags = []
        t_calls = 0.0
        b = draw()
        while True:
            now = time.perf_counter()
            if now - t0 > duration:
                break
            if rate is None or now >= next_t:
                c0 = time.perf_counter()
                tk = srv.submit(*b)
                t_calls += time.perf_counter() - c0
                if tk is None:  # admission full: wait for the oldest, then retry the same batch
                    busy += 1
                    if pending:
                        srv.wait(pending.pop(0))
                    continue
                if rate is not None:
                    lags.append(now - next_t)  # how late the host submitted it
                pending.append(tk)
                n_sub += 1
                b = draw()
                if rate is not None:
                    next_t += rng.exponential(1.0 / rate)
            else:
                c0 = time.perf_counter()
                while pending and srv.poll(pending[0]):
                    pending.pop(0)
                t_calls += time.perf_counter() - c0
                time.sleep(min(0.0002, max(0.0, next_t - now)))
        for tk in pending:
            srv.wait(tk)
        st = srv.stats(reset=False)
        lags.sort()
        st["host"] = {"submits": n_sub, "busy_refusals": busy, "call_s": t_calls,
                      "p50_submit_lag_ms": lags[len(lags) // 2] * 1e3 if lags else 0.0,
                      "max_submit_lag_ms": lags[-1] * 1e3 if lags else 0.0}
        return st, n_sub

    run(seconds / 2, None)  # warm-up: the first pass inserts the pools' new keys (the tree grows once)
    cap, _ = run(seconds, None)
    mean_batch = (2.0 ** 22 - 2.0 ** 10) / np.log(2.0 ** 12)  # mean of the log-uniform size law
    out = {"capacity_mops": cap["mops"], "capacity_device_mops": cap["device_mops"], "capacity_batches": cap["batches"],
           "policy": policy}
    res = {}
    sustainable = 0.0
    for frac in sorted(set(loads) | {load}):
        rate = frac * cap["mops"] * 1e6 / mean_batch
        s0 = tree.stats()  # (waits for the persistent kernel's idle exit: counters are flushed then)
        lat, n_sub = run(seconds, rate)
        s1 = tree.stats()
        offered = rate * mean_batch / 1e6
        res[f"{int(round(frac * 100))}%"] = {
            "offered_batches_per_s": rate, "offered_mops": offered, "mops": lat["mops"], "batches": lat["batches"],
            "p50_batch_ms": lat["p50_ms"], "p99_batch_ms": lat["p99_ms"], "max_batch_ms": lat["max_ms"],
            "p50_service_ms": lat["p50_service_ms"], "p99_service_ms": lat["p99_service_ms"],
            "device_mops": lat["device_mops"], "kernel_launches": lat["kernel_launches"],
            "stm_commits": s1["commits"] - s0["commits"], "stm_aborts": s1["aborts"] - s0["aborts"],
            "retry_exhausted": s1["retry_exhausted"] - s0["retry_exhausted"], "host": lat["host"]}
        if lat["mops"] >= 0.95 * offered and lat["p99_ms"] <= 10 * max(lat["p50_ms"], 1e-9):
            sustainable = max(sustainable, offered)
    srv.stop()
    head = res[f"{int(round(load * 100))}%"]
    out.update({k: head[k] for k in ("offered_batches_per_s", "offered_mops", "mops", "batches", "p50_batch_ms",
                                     "p99_batch_ms", "max_batch_ms", "kernel_launches")})
    out["sustainable_mops"] = sustainable
    out["loads"] = res
    out["workload"] = ("batch sizes log-uniform 2^10..2^22, search fraction U[0.5,1] per batch, Poisson arrivals "
                       "at fractions of the saturated rate (top-level figures: 50%); latency = submit to answers "
                       "in host memory; service = device time from the first claimed chunk to the last")
    return out


def run_stm_only(args):
    """BT_MODE_STM batches only (one GPU): a 2^tree-log2-key tree, --warmup
    then --steps batches of 2^batch-log2 requests (--search-pct GETs), timed
    with CUDA events; reports Mops/s and the STM counters."""
    import torch

    import eirene_b200 as E

    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream()
    n_tree, n_b = 1 << args.tree_log2, 1 << args.batch_log2
    tree = E.BTree(max_keys=2 * n_tree + 32 * n_b, max_batch=n_b, search_group=args.search_group)
    tree.set_option(E.OPT_STM_COMBINE, 0 if args.no_stm_combine else 1)
    tk = torch.empty(n_tree, dtype=torch.int64, device="cuda")
    tv = torch.empty(n_tree, dtype=torch.int64, device="cuda")
    E.gen_keys(args.dist, 1, n_tree, tk, tv, stream)
    tree.bulk_build(tk, tv, stream)
    del tv
    out = {"workload": f"BT_MODE_STM batches of 2^{args.batch_log2} requests, {args.search_pct}% search, "
                       f"on a 2^{args.tree_log2}-key {args.dist} tree",
           "stm_combine": not args.no_stm_combine}
    out.update(stm_run(E, torch, tree, tk, n_b, args.warmup, args.steps, args.dist, args.search_pct, 80_000, stream))
    print(json.dumps(out), flush=True)
    tree.close()
    return 0


def run_serve_only(args):
    """Serving only (one GPU): a 2^tree-log2-key tree, then serve_bench for
    the --descent form(s) with --serve-policy."""
    import numpy as np
    import torch

    import eirene_b200 as E

    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream()
    n_tree = 1 << args.tree_log2
    pool = (1 << args.pool_keys_log2) if args.pool_keys_log2 else 2 * n_tree + (32 << 22)
    tree = E.BTree(max_keys=pool, max_batch=1 << 22, search_group=args.search_group)
    tk = torch.empty(n_tree, dtype=torch.int64, device="cuda")
    tv = torch.empty(n_tree, dtype=torch.int64, device="cuda")
    E.gen_keys(args.dist, 1, n_tree, tk, tv, stream)
    tree.bulk_build(tk, tv, stream)
    del tv
    out = {"workload": f"serving on a 2^{args.tree_log2}-key {args.dist} tree"}
    forms = ["plain", "learned"] if args.descent == "both" else [args.descent]
    for form in forms:
        if form == "learned":
            tree.retrain(stream)
        tree.set_descent(form == "learned")
        out[form] = serve_bench(E, np, tree, tk, n_tree, seconds=args.serve_seconds, seed=5,
                                policy=args.serve_policy)
    print(json.dumps(out), flush=True)
    tree.close()
    return 0


# ----------------------------------------------------------------------------
def oracle_check(args, n_b, check_out, tk, draw):
    """Replays batches through the CPU oracle in the order the GPU ran them
    and compares the first timed batch of each run request by request.  Each
    run (a form's one-call-per-batch run, and its bt_execute_batches run)
    starts from the freshly built tree, as on the GPU, and its warm-up
    batches come first.  The batches are drawn again by the device
    generator, which is deterministic (`draw(seed)` returns host arrays), and
    copied to the host one at a time; the tree keys are the device's `tk`."""
    import numpy as np

    from oracle import oracle as O

    threads = os.cpu_count() or 1
    t0 = time.time()
    keys = tk.cpu().numpy().view(np.uint64)
    vals = O.value_of(keys)
    engine = O.ENGINE_MERGE if args.engine == "merge" else O.ENGINE_STM
    out = {}
    for run, (seed0, gv, gs) in check_out.items():
        tree = O.OracleTree(24, 24)
        tree.bulk_build(keys, vals)
        for i in range(args.warmup + 1):
            rk, rv, ro = draw(seed0 + i)
            ov, os_ = tree.execute_merged(rk, rv, ro, engine, threads)
            if i == args.warmup:
                bad = int(((ov != gv) | (os_ != gs)).sum())
                out[run] = {"requests": n_b, "mismatches": bad}
        del tree
    out["oracle_s"] = time.time() - t0
    out["batch"] = ("first timed batch of each run (forms one call per batch; *_pipelined: bt_execute_batches), "
                    "answers (value + status) per request")
    return out


def run_lookups(args):
    """Unsorted point lookups only (one GPU): build a 2^tree-log2 tree, train
    the model when the learned form is asked for, then time `steps` calls of
    bt_search_batch over 2^batch-log2 keys (half present) per form."""
    import torch

    import eirene_b200 as E

    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream()
    n_tree, n_b = 1 << args.tree_log2, 1 << args.batch_log2
    pool = (1 << args.pool_keys_log2) if args.pool_keys_log2 else 2 * n_tree
    tree = E.BTree(max_keys=pool, max_batch=n_b, search_group=args.search_group)
    tk = torch.empty(n_tree, dtype=torch.int64, device="cuda")
    tv = torch.empty(n_tree, dtype=torch.int64, device="cuda")
    E.gen_keys(args.dist, 1, n_tree, tk, tv, stream)
    tree.bulk_build(tk, tv, stream)
    del tv
    qk = torch.empty(n_b, dtype=torch.int64, device="cuda")
    qv = torch.empty(n_b, dtype=torch.int64, device="cuda")
    qo = torch.empty(n_b, dtype=torch.uint8, device="cuda")
    E.gen_requests(args.dist, 40_000, tk, n_b, 100, qk, qv, qo, stream)
    ov = torch.empty(n_b, dtype=torch.int64, device="cuda")
    ost = torch.empty(n_b, dtype=torch.uint8, device="cuda")
    out = {"workload": f"unsorted lookups of 2^{args.batch_log2} keys (half present) in a 2^{args.tree_log2}-key "
                       f"{args.dist} tree", "steps": args.steps, "warmup": args.warmup}
    forms = ["plain", "learned"] if args.descent == "both" else [args.descent]
    for form in forms:
        if form == "learned":
            tree.retrain(stream)
        tree.set_descent(form == "learned")
        tune = None if args.no_autotune else tree.autotune(qk, stream)
        for _ in range(args.warmup):
            tree.search(qk, ov, ost, stream)
        tree.reset_stats()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            tree.search(qk, ov, ost, stream)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
        st = tree.stats()
        out[form] = {"mops": n_b / ms / 1e3, "ms_per_call": ms,
                     "dram_alg_gbs": BYTES_SEARCH * n_b / ms / 1e6,
                     "learned_fallbacks": st["learned_fallbacks"], "learned_hits": st["learned_hits"],
                     "autotune": tune}
    print(json.dumps(out), flush=True)
    tree.close()
    return 0


def unique_op_counts(torch, k, o):
    """(unique GET keys, unique INSERT keys) of a batch under the merged meaning."""
    u, inv = torch.unique(k, return_inverse=True)
    has_ins = torch.zeros(u.numel(), dtype=torch.int32, device=k.device)
    has_ins.scatter_reduce_(0, inv, (o == 0).to(torch.int32), reduce="amax")
    n_ins = int(has_ins.sum().item())
    return u.numel() - n_ins, n_ins


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--tree-log2", type=int, default=26)
    ap.add_argument("--batch-log2", type=int, default=22)
    ap.add_argument("--search-pct", type=int, default=95)
    ap.add_argument("--dist", default="uniform", choices=["uniform", "zipf", "normal", "gamma"])
    ap.add_argument("--descent", default="both", choices=["plain", "learned", "both"])
    ap.add_argument("--search-group", type=int, default=4)
    ap.add_argument("--segments", type=int, default=0,
                    help="learned predictor segments (0: one per 64 leaves at training, at least 4096)")
    ap.add_argument("--engine", default="merge", choices=["merge", "stm"],
                    help="insert engine of the sorted batch: segmented leaf merge or warp STM")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-sample-log2", type=int, default=20)
    ap.add_argument("--no-serve", action="store_true")
    ap.add_argument("--serve-seconds", type=float, default=1.5)
    ap.add_argument("--retrain-every", type=int, default=0,
                    help="learned form: retrain the model after every K timed batches (0: trained once, before)")
    ap.add_argument("--retrain-mode", default="refit", choices=["refit", "full"],
                    help="retraining inside the timed region: refit (leaf array and segment lines follow the "
                         "leaves, stage 1 kept) or full (stage 1 trained again from its initial parameters)")
    ap.add_argument("--front-end", default="hash", choices=["hash", "sort"],
                    help="sorted batches: hash front end (sort only INSERT-coupled requests) or full sort")
    ap.add_argument("--pool-keys-log2", type=int, default=0,
                    help="size the node pool for 2^x keys (default: 2 x tree + 32 x batch)")
    ap.add_argument("--no-fill-tune", action="store_true",
                    help="build with the default node fill (24) instead of the fill autotuner's pick")
    ap.add_argument("--no-stm-pass", action="store_true",
                    help="skip the BT_MODE_STM passes (headline tree and a skewed Zipf tree) with abort counts")
    ap.add_argument("--no-same-box", action="store_true",
                    help="skip the comparison with the reference's GPU build on its own 31-bit benchmark shape")
    ap.add_argument("--serve-only", action="store_true",
                    help="run only the serving benchmark (continuous batching) on a 2^tree-log2-key tree")
    ap.add_argument("--serve-policy", type=int, default=0, choices=[0, 1],
                    help="serving: which admitted batch a free warp takes work from (0 oldest, 1 fewest unclaimed)")
    ap.add_argument("--check", action="store_true",
                    help="compare the answers of each form's first timed batch with the CPU oracle, which "
                         "replays every batch of the run before it (outside the timed region; one GPU)")
    ap.add_argument("--lookups-only", action="store_true",
                    help="time only unsorted point lookups (bt_search_batch) of 2^batch-log2 keys, half present, "
                         "with the --descent form(s); a small, bounded workload for kernel profiles")
    ap.add_argument("--no-autotune", action="store_true",
                    help="--lookups-only: keep the default launch shapes (no autotuner launches before timing)")
    ap.add_argument("--stm-only", action="store_true",
                    help="time only BT_MODE_STM batches (v39 meaning) of 2^batch-log2 requests on a "
                         "2^tree-log2-key --dist tree, requests drawn from the same law; a bounded workload for "
                         "kernel profiles")
    ap.add_argument("--touch-sort", choices=["auto", "merge", "radix"], default="auto",
                    help="sort of the requests a write touches (BT_OPT_TOUCH_SORT): by the touched count seen "
                         "last (default), always the tile sort plus merge rounds, always the onesweep radix sort")
    ap.add_argument("--no-host-front-overlap", action="store_true",
                    help="e2e: run each host batch whole on the stream (BT_OPT_HOST_FRONT_OVERLAP 0) instead of "
                         "its front part beside the previous host batch's tree part")
    ap.add_argument("--no-stm-combine", action="store_true",
                    help="--stm-only: run every INSERT as its own transaction (BT_OPT_STM_COMBINE 0)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3

    if args.impl == "reference":
        return run_reference(args)
    if args.lookups_only:
        return run_lookups(args)
    if args.serve_only:
        return run_serve_only(args)
    if args.stm_only:
        return run_stm_only(args)

    import numpy as np
    import torch

    import eirene_b200 as E

    rank, world, local = env_int("RANK", 0), env_int("WORLD_SIZE", 1), env_int("LOCAL_RANK", 0)
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def allmax(x: float) -> float:
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def allsum(x: int) -> int:
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.int64, device="cuda")
        dist.all_reduce(t)
        return int(t.item())

    n_tree = 1 << args.tree_log2
    n_b = 1 << args.batch_log2
    n_steps_total = args.warmup + args.steps
    stream = torch.cuda.current_stream()
    # ---- tree
    pool_keys = (1 << args.pool_keys_log2) if args.pool_keys_log2 else 2 * n_tree + 32 * n_b
    sharded = None
    if world > 1:
        from eirene_b200.shard import ShardedBTree

        # an owner receives about n_b requests per step; headroom keeps that one local batch
        sharded = ShardedBTree.on_gpu(max_keys=pool_keys, max_batch=n_b + n_b // 8, device=local,
                                      search_group=args.search_group, n_segments=args.segments)
        tree = sharded.ops.tree
    else:
        tree = E.BTree(max_keys=pool_keys, max_batch=n_b, device=local, search_group=args.search_group,
                       n_segments=args.segments)
    tree.set_option(E.OPT_FRONT_END, 1 if args.front_end == "hash" else 0)
    tree.set_option(E.OPT_HOST_FRONT_OVERLAP, 0 if args.no_host_front_overlap else 1)
    tree.set_option(E.OPT_TOUCH_SORT, {"radix": 0, "merge": 1, "auto": 2}[args.touch_sort])
    tk = torch.empty(n_tree, dtype=torch.int64, device="cuda")
    tv = torch.empty(n_tree, dtype=torch.int64, device="cuda")
    E.gen_keys(args.dist, 1 + rank, n_tree, tk, tv, stream)
    # node fill (fanout) from the autotuner, on a sample tree of 2^22 of the
    # keys, before the tree is built (later splits use it too)
    fill = None
    if sharded is None and not args.no_fill_tune:
        fill = tree.autotune_fill(tk[: min(n_tree, 1 << 22)], stream)
    def build_tree(tv):
        if sharded is not None:
            sharded.bulk_build(tk, tv)
        else:
            tree.bulk_build(tk, tv, stream)

    t0 = time.time()
    build_tree(tv)
    torch.cuda.synchronize()
    build_s = time.time() - t0
    del tv
    built = [True]  # the tree as bulk-built, no batch applied yet

    def rebuild_tree():
        # each form starts from the same freshly built tree: the batches of
        # the form measured first must not grow the other form's tree
        if built[0]:
            return
        tv = torch.empty(n_tree, dtype=torch.int64, device="cuda")
        E.gen_keys(args.dist, 1 + rank, n_tree, tk, tv, stream)
        build_tree(tv)
        torch.cuda.synchronize()
        del tv
        built[0] = True

    # ---- batches: distinct, device resident (each step reads its own 2^22-request batch)
    def make_batches(seed0):
        out = []
        for i in range(n_steps_total):
            k = torch.empty(n_b, dtype=torch.int64, device="cuda")
            v = torch.empty(n_b, dtype=torch.int64, device="cuda")
            o = torch.empty(n_b, dtype=torch.uint8, device="cuda")
            E.gen_requests(args.dist, seed0 + 1000 * rank + i, tk, n_b, args.search_pct, k, v, o, stream)
            out.append((k, v, o))
        torch.cuda.synchronize()
        return out

    ov = torch.empty(n_b, dtype=torch.int64, device="cuda")
    ost = torch.empty(n_b, dtype=torch.uint8, device="cuda")
    MODE = E.MODE_SORTED | (E.MODE_MERGE_ENGINE if args.engine == "merge" else 0)

    def step(k, v, o, out=None):
        a, b = out if out is not None else (ov, ost)
        if sharded is not None:
            sharded.execute(k, v, o, a, b, mode=MODE)
        else:
            tree.execute(k, v, o, a, b, mode=MODE, stream=stream)

    # --check: the first timed batch of each form answers into its own
    # buffers (no extra work in the timed region); the oracle replays the
    # same seeded batches afterwards and compares
    check_out = {}

    def run_form(learned: bool, seed0: int):
        rebuild_tree()
        built[0] = False
        batches = make_batches(seed0)
        counts = [unique_op_counts(torch, k, o) for (k, v, o) in batches[args.warmup:]]
        info = None
        if learned:
            t_r = time.time()
            tree.retrain(stream)
            info = tree.learned_info()
            info["retrain_s"] = time.time() - t_r
            tree.set_descent(True)
        else:
            tree.set_descent(False)
        # autotune lane counts / leaf loads on this tree with the first batch's keys,
        # then pin the batch descent to the form being measured
        tune = tree.autotune(batches[0][0], stream)
        tree.set_option(E.OPT_BATCH_DESCENT, 1 if learned else 0)
        for i in range(args.warmup):
            step(*batches[i])
        tree.reset_stats()
        tree.profile(True)
        tree.profile_read(reset=True)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 2)]
        barrier()
        sampler = ClockSampler(local)
        sampler.start()
        l0 = E.launch_count()
        ev[0].record(stream)
        first = None
        if args.check:
            first = (torch.empty(n_b, dtype=torch.int64, device="cuda"),
                     torch.empty(n_b, dtype=torch.uint8, device="cuda"))
        for s in range(args.steps):
            step(*batches[args.warmup + s], out=first if s == 0 else None)
            if learned and args.retrain_every > 0 and (s + 1) % args.retrain_every == 0:
                # inside the timed region: the model follows the tree
                if args.retrain_mode == "refit":
                    tree.refit(stream)
                else:
                    tree.retrain(stream)
            ev[s + 1].record(stream)  # the batch's answers are final
        tree.sync(stream)  # the last batch's deferred leaf/inner merge
        ev[-1].record(stream)
        torch.cuda.synchronize()
        launches = E.launch_count() - l0
        clocks = sampler.stop()
        barrier()
        step_ms = [ev[s].elapsed_time(ev[s + 1]) for s in range(args.steps)]
        total_ms = ev[0].elapsed_time(ev[-1])  # up to the end of every batch's write phase
        phases = tree.profile_read(reset=True)
        tree.profile(False)
        st = tree.stats()
        if first is not None:
            check_out["learned" if learned else "plain"] = (seed0, first[0].cpu().numpy().view(np.uint64),
                                                            first[1].cpu().numpy())
        del batches
        pipe = None
        if sharded is None:
            # throughput through bt_execute_batches: fresh batches of the same
            # kind, each with its own answer arrays, on a freshly built tree
            # (and model), batch j + 1's front part beside batch j's tree part;
            # a --retrain-every schedule runs as chunks with the refit between
            rebuild_tree()
            built[0] = False
            tree.set_descent(False)
            if learned:
                tree.retrain(stream)
                tree.set_descent(True)
            tree.set_option(E.OPT_BATCH_DESCENT, 1 if learned else 0)
            batches = make_batches(seed0 + 500)
            outs = [(torch.empty(n_b, dtype=torch.int64, device="cuda"),
                     torch.empty(n_b, dtype=torch.uint8, device="cuda")) for _ in batches]
            tree.execute_many(batches[:args.warmup], outs[:args.warmup], mode=MODE, stream=stream)
            tree.sync(stream)
            torch.cuda.synchronize()
            tree.reset_stats()
            barrier()
            sampler = ClockSampler(local)
            sampler.start()
            l0 = E.launch_count()
            p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            K = args.retrain_every if (learned and args.retrain_every > 0) else args.steps
            p0.record(stream)
            for c0 in range(args.warmup, args.warmup + args.steps, K):
                c1 = min(c0 + K, args.warmup + args.steps)
                tree.execute_many(batches[c0:c1], outs[c0:c1], mode=MODE, stream=stream)
                if K < args.steps and (c1 - args.warmup) % K == 0:
                    if args.retrain_mode == "refit":
                        tree.refit(stream)
                    else:
                        tree.retrain(stream)
            tree.sync(stream)
            p1.record(stream)
            torch.cuda.synchronize()
            pipe = {"total_ms": p0.elapsed_time(p1), "launches": E.launch_count() - l0, "clocks": sampler.stop(),
                    "stats": tree.stats()}
            if args.check:
                a, b = outs[args.warmup]
                check_out[("learned" if learned else "plain") + "_pipelined"] = (
                    seed0 + 500, a.cpu().numpy().view(np.uint64), b.cpu().numpy())
            barrier()
            del batches, outs
        return {"total_ms": total_ms, "step_ms": step_ms, "phases": phases, "counts": counts,
                "launches": launches, "clocks": clocks, "stats": st, "learned_info": info, "tune": tune,
                "pipe": pipe}

    forms = {}
    if args.descent in ("plain", "both"):
        forms["plain"] = run_form(False, 10_000)
    if args.descent in ("learned", "both"):
        try:
            forms["learned"] = run_form(True, 20_000)
        except E.BTError as e:
            forms["learned_error"] = str(e)
    # headline: the faster of the two forms (both are reported under "forms")
    cands = [f for f in ("plain", "learned") if f in forms]
    def form_ms(F):  # the throughput run: bt_execute_batches when it ran, else one call per batch
        return F["pipe"]["total_ms"] if F.get("pipe") else F["total_ms"]

    head = min(cands, key=lambda f: form_ms(forms[f]))
    R = forms[head]

    # unsorted point lookups (bt_search_batch on random keys): plain vs learned
    random_lookup = {}
    try:
        if sharded is not None:
            raise E.BTError(-1, "per-GPU lookups are measured at n_gpus=1")
        rk = torch.empty(n_b, dtype=torch.int64, device="cuda")
        rv = torch.empty(n_b, dtype=torch.int64, device="cuda")
        ro = torch.empty(n_b, dtype=torch.uint8, device="cuda")
        E.gen_requests(args.dist, 40_000 + rank, tk, n_b, 100, rk, rv, ro, stream)
        for form in ("plain", "learned"):
            if form == "learned" and "learned" not in forms:
                continue
            if form == "learned":
                tree.refit(stream)  # the model follows the tree the batches grew
            tree.set_descent(form == "learned")
            for _ in range(3):
                tree.search(rk, ov, ost, stream)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(5):
                tree.search(rk, ov, ost, stream)
            e1.record(stream)
            torch.cuda.synchronize()
            random_lookup[form] = n_b * 5 / (e0.elapsed_time(e1) / 1e3) / 1e6
        del rk, rv, ro
    except E.BTError as ex:
        random_lookup["error"] = str(ex)
    total_ms = allmax(form_ms(R))
    value = world * n_b * args.steps / (total_ms / 1e3) / 1e6

    # ---- roofline of the dominant phase
    hbm, peak_kind = peaks()
    steps = args.steps
    ph = R["phases"]
    n_get = sum(c[0] for c in R["counts"]) / steps
    n_ins = sum(c[1] for c in R["counts"]) / steps
    alg = {"sort": BYTES_SORT * n_b, "search": BYTES_SEARCH * n_get, "insert": BYTES_INSERT * n_ins}
    # with the hash front end the "sort" and "merge" phases are spans of a side
    # stream that overlap the lookups, not kernels of their own
    cand = ("search", "insert", "writeback") if args.front_end == "hash" else ("sort", "merge", "search", "insert",
                                                                              "writeback")
    dom = max(cand, key=lambda p: ph[p])
    dom_ms = ph[dom] / max(1, ph["batches"])
    dom_bytes = alg.get(dom)
    traffic = None
    # DRAM bytes per unit of the dominant kernel from an ncu capture, kept as a
    # "bytes_per_unit: N" line in profiles/traffic_<phase>.md
    tpath = os.path.join(ROOT, "profiles", f"traffic_{dom}.md")
    if head == "learned" and dom == "search":  # the learned form's lookup kernel
        tpath = os.path.join(ROOT, "profiles", "traffic_search_learned.md")
    if os.path.exists(tpath):
        try:
            import re

            m = re.search(r"bytes_per_unit:\s*([0-9.]+)", open(tpath).read())
            if m:
                traffic = float(m.group(1)) * (n_get if dom == "search" else n_ins if dom == "insert" else n_b)
        except Exception:
            traffic = None
    roof = None
    if dom_bytes:
        ach = dom_bytes / (dom_ms / 1e3) / 1e9
        kname = dom
        if dom == "search":
            tune = R.get("tune") or {}
            if head == "learned":
                m, g = tune.get("learned_mode", 3), tune.get("learned_lanes", 4)
                kname = (f"search phase: learned_pipe_kernel<{g}> + search2_kernel over its misses" if m == 3 else
                         f"search phase: learned_lookup_kernel<{g},{m}> + search2_kernel over its misses")
            else:
                kname = f"search phase: search2_kernel<{tune.get('plain_lanes', 4)},0,1>"
        roof = {"kernel": kname, "bound": "hbm", "achieved": ach, "peak": hbm, "unit": "GB/s", "frac": ach / hbm,
                "peak_source": peak_kind, "traffic": traffic, "alg_bytes_per_launch": dom_bytes,
                "launch_ms": dom_ms}

    # ---- e2e through the host entry point (pinned host buffers, copies timed),
    # with the headline form's descent
    e2e = None
    tree.set_descent(head == "learned")
    tree.set_option(E.OPT_BATCH_DESCENT, 1 if head == "learned" else 0)
    if True:
        hb = []
        # 30 steps: the first batch's copy-in and the last one's copy-out
        # overlap nothing (about 1.4 ms per run), spread over the steps
        e2e_steps = 30
        # page-locked host buffers from the library's own allocator (bt_host_alloc)
        pinned = []

        def host_buf(n, dtype):
            b = E.HostBuffer(n, dtype)
            pinned.append(b)
            return b.tensor

        # pinned host batches, refilled with fresh requests before each timed
        # loop: a loop that replayed batches the tree had already applied would
        # time INSERTs that are all updates of existing keys
        dk = torch.empty(n_b, dtype=torch.int64, device="cuda")
        dv = torch.empty(n_b, dtype=torch.int64, device="cuda")
        do = torch.empty(n_b, dtype=torch.uint8, device="cuda")
        for i in range(1 + e2e_steps):
            hb.append((host_buf(n_b, torch.int64), host_buf(n_b, torch.int64), host_buf(n_b, torch.uint8),
                       host_buf(n_b, torch.int64)))
        n_ins = [0] * (1 + e2e_steps)

        def fill_host(seed0):
            for i, (hk, hv, ho, hiv) in enumerate(hb):
                E.gen_requests(args.dist, seed0 + 1000 * rank + i, tk, n_b, args.search_pct, dk, dv, do, stream)
                torch.cuda.synchronize()
                hk.copy_(dk)
                hv.copy_(dv)
                ho.copy_(do)
                # the same batch with the INSERTs' values only, packed in request order
                iv = dv[do == E.OP_INSERT]
                hiv[: iv.numel()].copy_(iv)
                n_ins[i] = iv.numel()

        # three answer buffers: three batches in flight (the handle's three
        # staging sets): batch s is submitted once batch s - 3 is answered
        outs = [(host_buf(n_b, torch.int64), host_buf(n_b, torch.uint8)) for _ in range(3)]

        def host_submit(i, out, packed):
            k, v, o, iv = hb[i]
            iv = iv[: n_ins[i]]
            hov, hos = out
            if sharded is not None:
                # host batch in, host answers out, through the sharded tree
                dk.copy_(k, non_blocking=True)
                dv.copy_(v, non_blocking=True)
                do.copy_(o, non_blocking=True)
                sharded.execute(dk, dv, do, ov, ost, mode=MODE)
                hov.copy_(ov, non_blocking=True)
                hos.copy_(ost, non_blocking=True)
                return None
            # three batches in flight: the next batch's copy-in and the
            # previous batch's copy-out beside this batch's kernels
            if packed:  # bt_execute_batch_host_packed_async
                return tree.submit_host_packed(k, o, iv, hov, hos, mode=MODE, stream=stream)
            return tree.submit_host(k, v, o, hov, hos, mode=MODE, stream=stream)  # bt_execute_batch_host_async

        def host_wait(t):
            if t is not None:
                tree.wait_host(t)

        def timed(packed, seed0):
            # like the device-resident forms: a freshly built tree, the
            # headline form's model trained on it
            rebuild_tree()
            built[0] = False
            tree.set_descent(False)
            if head == "learned":
                tree.retrain(stream)
            tree.set_descent(head == "learned")
            tree.set_option(E.OPT_BATCH_DESCENT, 1 if head == "learned" else 0)
            fill_host(seed0)
            for _ in range(3):
                host_wait(host_submit(0, outs[0], packed))
            barrier()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            w0 = time.perf_counter()
            e0.record(stream)
            tickets = []
            for s in range(e2e_steps):
                if s >= 3:
                    host_wait(tickets[s - 3])
                tickets.append(host_submit(1 + s, outs[s % 3], packed))
            for t in tickets[-3:]:
                host_wait(t)
            tree.sync(stream)
            e1.record(stream)
            torch.cuda.synchronize()
            wall_ms = (time.perf_counter() - w0) * 1e3
            barrier()
            return allmax(e0.elapsed_time(e1)), wall_ms

        packed = sharded is None
        e2e_ms, wall_ms = timed(True, 50_000) if packed else (None, None)
        full_ms, full_wall = timed(False, 30_000)
        if not packed:
            e2e_ms, wall_ms = full_ms, full_wall
        del hb, outs
        for b in pinned:
            b.free()
        # bytes over the bus per step: keys and op codes copied in with the
        # INSERTs' values (packed) or every request's value slot; values and
        # status bytes copied out
        ins_per_step = sum(n_ins[1:]) / e2e_steps
        e2e = {"value": world * n_b * e2e_steps / (e2e_ms / 1e3) / 1e6, "unit": "Mops/s",
               "h2d_bytes_per_step": int(n_b * 9 + 8 * ins_per_step) if packed else n_b * 17,
               "d2h_bytes_per_step": n_b * 9,
               "host_wall_ms_per_step": wall_ms / e2e_steps,
               "pipelined": sharded is None,
               "front_overlap": sharded is None and not args.no_host_front_overlap,
               "entry_point": "bt_execute_batch_host_packed_async" if packed else "sharded execute",
               "steps": e2e_steps, "descent": head,
               "full_values": {"value": world * n_b * e2e_steps / (full_ms / 1e3) / 1e6,
                               "entry_point": "bt_execute_batch_host_async",
                               "h2d_bytes_per_step": n_b * 17, "d2h_bytes_per_step": n_b * 9,
                               "host_wall_ms_per_step": full_wall / e2e_steps}}

    serving = {}
    if not args.no_serve and sharded is None:
        for form in ("plain", "learned"):
            if form == "learned" and "learned" not in forms:
                continue
            try:
                tree.set_descent(form == "learned")
                serving[form] = serve_bench(E, np, tree, tk, n_tree, seconds=args.serve_seconds, seed=5 + rank,
                                            policy=args.serve_policy)
            except Exception as ex:  # reported, not fatal
                serving[form] = {"error": str(ex)}

    stm = None
    if world == 1 and not args.no_stm_pass:
        try:
            stm = stm_passes(E, torch, tree, tk, n_b, 5, args.search_pct, stream)
        except Exception as ex:  # reported, not fatal
            stm = {"error": str(ex)}
    same_box = None
    if not args.no_same_box and world == 1:
        try:
            same_box = same_box_ours(E, torch)
        except Exception as ex:  # reported, not fatal
            same_box = {"error": str(ex)}

    launches = allsum((R["pipe"] or R)["launches"])
    check = None
    if args.check and world == 1 and check_out:
        def draw(seed):
            k = torch.empty(n_b, dtype=torch.int64, device="cuda")
            v = torch.empty(n_b, dtype=torch.int64, device="cuda")
            o = torch.empty(n_b, dtype=torch.uint8, device="cuda")
            E.gen_requests(args.dist, seed, tk, n_b, args.search_pct, k, v, o, stream)
            torch.cuda.synchronize()
            return k.cpu().numpy().view(np.uint64), v.cpu().numpy().view(np.uint64), o.cpu().numpy()

        check = oracle_check(args, n_b, check_out, tk, draw)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_baseline(args, 1 << args.cpu_sample_log2, os.cpu_count() or 1)
        except Exception as ex:  # reported, not fatal
            cpu = {"error": str(ex)}

    if rank == 0:
        def form_summary(F):
            ms = sorted(F["step_ms"])
            tot = F["total_ms"]
            s = F["stats"]
            P = F.get("pipe")
            ptot = form_ms(F)
            return {
                "value": n_b * steps / (ptot / 1e3) / 1e6, "ms_per_step": ptot / steps,
                "p50_batch_ms": ms[len(ms) // 2], "p99_batch_ms": ms[min(len(ms) - 1, int(0.99 * len(ms)))],
                "per_call": {"value": n_b * steps / (tot / 1e3) / 1e6, "ms_per_step": tot / steps},
                "pipelined": ({"learned_hits": P["stats"]["learned_hits"],
                               "learned_fallbacks": P["stats"]["learned_fallbacks"]} if P else None),
                "phases_ms_per_step": {p: F["phases"][p] / max(1, F["phases"]["batches"])
                                       for p in ("sort", "merge", "search", "insert", "writeback")},
                "stm_aborts": s["aborts"], "stm_commits": s["commits"],
                "learned_hits": s["learned_hits"], "learned_fallbacks": s["learned_fallbacks"],
                "mean_probe": s["learned_probe_sum"] / max(1, s["learned_hits"]),
                "model": F.get("learned_info"),
                "autotune": F.get("tune"),
            }

        line = {
            "metric": METRIC, "value": value, "unit": "Mops/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "config": {
                "workload": f"2^{args.tree_log2} {args.dist} uint64 keys per GPU, batches of 2^{args.batch_log2} "
                            f"requests, {args.search_pct}% search / {100 - args.search_pct}% insert, "
                            f"sort-merged (v38 meaning), {args.front_end} front end, {args.engine} insert engine",
                "descent": head, "tree_keys": n_tree, "batch": n_b, "search_group": args.search_group,
                "l2": "inputs larger than L2: tree ~1.5 GB; every step reads its own 71 MB batch",
                "parallelism": (f"{world} key-range shards, one tree per GPU, all-to-all request exchange over NCCL"
                                if sharded is not None else "one tree on one GPU"),
                "tree_build_s": build_s,
                "learned_retrain_every": args.retrain_every,
                "node_fill": fill,
                "learned_retrain_mode": args.retrain_mode,
                "touch_sort": args.touch_sort,
                "throughput": ("bt_execute_batches over the timed batches (batch j + 1's front part beside batch "
                               "j's lookups and writes); p50 / p99 batch latency and phases: the same kind of "
                               "batches, one bt_execute_batch call each (forms.*.per_call)"
                               if R.get("pipe") else "one bt_execute_batch call per batch"),
            },
            "roofline": roof,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "clocks": (R["pipe"] or R)["clocks"],
            "gpu_launches": launches,
            "p50_batch_ms": form_summary(R)["p50_batch_ms"],
            "p99_batch_ms": form_summary(R)["p99_batch_ms"],
            "forms": {k: form_summary(v) for k, v in forms.items() if isinstance(v, dict)},
            "random_lookup_mops": random_lookup,
            "serving": serving,
        }
        if "learned_error" in forms:
            line["learned_error"] = forms["learned_error"]
        if check is not None:
            line["check"] = check
        if same_box is not None:
            line["same_box_31bit"] = same_box
        if stm is not None:
            line["stm"] = stm
        print(json.dumps(line), flush=True)
    tree.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
