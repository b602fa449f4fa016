"""Build the pentago_b200 CUDA library in-tree for sm_100a.

    python -m pentago_b200.build

Compiles every file under pentago_b200/csrc into pentago_b200/_lib/libpentago_b200.so
with nvcc (no PyTorch in the signatures; plain C ABI declared in include/pentago_b200.h).
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_lib")
LIB = os.path.join(OUT, "libpentago_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-Xptxas", "-warn-spills"]


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cc")))


def build(verbose=False, jobs=None):
    os.makedirs(OUT, exist_ok=True)
    objs, procs = [], []
    for src in sources():
        obj = os.path.join(OUT, os.path.basename(src) + ".o")
        objs.append(obj)
        deps = [src] + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
        deps.append(os.path.join(HERE, "..", "include", "pentago_b200.h"))
        if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(d) for d in deps):
            continue
        lang = ["-x", "cu"] if src.endswith(".cu") else ["-x", "c++"]
        cmd = [NVCC] + ARCH + FLAGS + lang + ["-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    failed = False
    for cmd, p in procs:
        out = p.communicate()[0].decode()
        if out.strip():
            print(out, end="" if out.endswith("\n") else "\n", file=sys.stderr)
        if p.returncode:
            failed = True
            print("FAILED: " + " ".join(cmd), file=sys.stderr)
    if failed:
        raise RuntimeError("nvcc failed")
    if not procs and os.path.exists(LIB):
        return LIB
    cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart_static", "-lrt", "-ldl", "-lpthread", "-lz"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
