"""Build libeirene_b200.so in place with nvcc for sm_100a.

The library is the product: hand-written CUDA kernels plus the C ABI declared
in include/eirene_b200.h.  It is built in-tree (eirene_b200/libeirene_b200.so)
so that it travels with the source tree; no JIT cache is involved.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libeirene_b200.so")
SOURCES = [
    "bt_sort.cu",
    "bt_tree.cu",
    "bt_stm.cu",
    "bt_batch.cu",
    "bt_learned.cu",
    "bt_api.cu",
    "bt_workload.cu",
    "bt_static.cu",
    "bt_tune.cu",
    "bt_merge.cu",
    "bt_serve.cu",
    "bt_shard.cu",
    "bt_front.cu",
    "bt_snapshot.cu",
    "bt_delete.cu",
]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(ROOT, "include", "eirene_b200.h")]
    deps += [os.path.join(HERE, "host", f) for f in os.listdir(os.path.join(HERE, "host"))]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False, extra: list[str] | None = None) -> str:
    if not force and not _stale():
        return LIB
    objdir = os.path.join(ROOT, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    flags = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
                    "-I", os.path.join(ROOT, "include")] + (extra or [])
    procs = []
    for src in SOURCES:
        obj = os.path.join(objdir, src.replace(".cu", ".o"))
        objs.append(obj)
        cmd = [nvcc(), "-c", os.path.join(CSRC, src), "-o", obj] + flags
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    failed = False
    for src, p in procs:
        out = p.communicate()[0].decode()
        if p.returncode != 0:
            failed = True
            sys.stderr.write(f"--- nvcc failed on {src}\n{out}\n")
        elif verbose and out.strip():
            print(out)
    if failed:
        raise RuntimeError("nvcc failed")
    tmp = LIB + ".tmp"
    cmd = [nvcc(), "-shared", "-o", tmp] + objs + ARCH + ["-lcudart"]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    build_cli()
    return LIB


CLI = os.path.join(HERE, "bt_stm_test")


def build_cli() -> str:
    """The reference-compatible command-line driver (g++, links the library)."""
    host = os.path.join(HERE, "host")
    cmd = ["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), "-I", "/usr/local/cuda/include",
           os.path.join(host, "gpu_btree.cpp"), os.path.join(host, "bt_stm_test.cpp"), "-o", CLI,
           "-L", HERE, "-leirene_b200", "-L", "/usr/local/cuda/lib64", "-lcudart", "-Wl,-rpath,$ORIGIN", "-Wl,-rpath,/usr/local/cuda/lib64"]
    subprocess.run(cmd, check=True)
    return CLI


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
