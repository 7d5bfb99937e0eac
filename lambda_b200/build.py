"""Builds the sm_100a library liblambda_gpu.so in-tree with nvcc.

    python -m lambda_b200.build          # build if sources changed
    python -m lambda_b200.build --force  # rebuild

The library is a plain C-ABI shared object (include/lambda_gpu.h); Python
loads it with ctypes (lambda_b200/_lib.py).  It is built in the package
directory so that it travels with the repository.
"""
import argparse
import hashlib
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "liblambda_gpu.so")
BUILD_DIR = os.path.join(HERE, "_build")

CU_SOURCES = ["lgpu_api.cu", "lgpu_kernels.cu", "lgpu_trace.cu", "lgpu_render_k4.cu", "lgpu_render_k8.cu",
              "lgpu_render_k16.cu", "lgpu_batch_k4.cu", "lgpu_batch_k8.cu", "lgpu_batch_k16.cu",
              "lgpu_adjoint_k4.cu", "lgpu_adjoint_k8.cu", "lgpu_adjoint_k16.cu",
              "lgpu_noalloc.cu", "lgpu_probe.cu", "lgpu_bvh_build.cu", "lgpu_layout_dev.cu"]
CPP_SOURCES = ["lgpu_layout.cpp", "lgpu_sah.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _digest(extra_flags):
    h = hashlib.sha256()
    # the sources, the ABI header and this file (its compiler flags)
    names = sorted(os.listdir(CSRC)) + ["../../include/lambda_gpu.h", "../build.py"]
    for n in names:
        p = os.path.normpath(os.path.join(CSRC, n))
        if os.path.isfile(p):
            h.update(n.encode())
            with open(p, "rb") as f:
                h.update(f.read())
    h.update(" ".join(extra_flags).encode())
    return h.hexdigest()


def build(force=False, verbose=False, extra_flags=()):
    """Compiles every CUDA and C++ source into liblambda_gpu.so."""
    extra_flags = list(extra_flags)
    stamp = os.path.join(BUILD_DIR, "stamp")
    digest = _digest(extra_flags)
    if not force and os.path.exists(OUT) and os.path.exists(stamp):
        with open(stamp) as f:
            if f.read().strip() == digest:
                return OUT
    os.makedirs(BUILD_DIR, exist_ok=True)
    inc = ["-I" + os.path.join(REPO, "include"), "-I" + CSRC]
    # -fmad=false: no multiply-add contraction, so every float operation
    # rounds as written.  Kernels instantiated for different job policies and
    # material specialisations then compute bit-identical paths (a batched
    # job equals its plain render), and the shading arithmetic matches the
    # reference's operation for operation except in the transcendental
    # functions.  Traversal spells out its roundings (__fadd_rn etc.) anyway.
    common = ["-O3", "-std=c++17", "-fmad=false", "-Xcompiler", "-fPIC", "-lineinfo"] + inc
    objs = []
    cmds = []
    for src in CU_SOURCES:
        obj = os.path.join(BUILD_DIR, src + ".o")
        cmds.append([nvcc()] + ARCH + common + extra_flags +
                    ["-Xptxas", "-v", "-c", os.path.join(CSRC, src), "-o", obj])
        objs.append(obj)
    for src in CPP_SOURCES:
        obj = os.path.join(BUILD_DIR, src + ".o")
        cmds.append([nvcc()] + common + extra_flags + ["-Xcompiler", "-pthread", "-x", "c++", "-c",
                                                       os.path.join(CSRC, src), "-o", obj])
        objs.append(obj)
    procs = [subprocess.Popen(c, stdout=subprocess.PIPE, stderr=subprocess.STDOUT) for c in cmds]
    logs = []
    for c, p in zip(cmds, procs):
        out, _ = p.communicate()
        logs.append(out.decode(errors="replace"))
        if p.returncode != 0:
            sys.stderr.write(" ".join(c) + "\n" + logs[-1])
            raise RuntimeError("nvcc failed")
    with open(os.path.join(BUILD_DIR, "ptxas.log"), "w") as f:
        f.write("\n".join(logs))
    if verbose:
        print("\n".join(logs))
    tmp = OUT + ".tmp"
    link = [nvcc()] + ARCH + ["-shared", "-o", tmp] + objs + ["-lcudart", "-lpthread"]
    r = subprocess.run(link, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)
    if r.returncode != 0:
        sys.stderr.write(r.stdout.decode(errors="replace"))
        raise RuntimeError("link failed")
    os.replace(tmp, OUT)
    with open(stamp, "w") as f:
        f.write(digest)
    return OUT


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    args = ap.parse_args()
    print(build(force=args.force, verbose=args.verbose))


if __name__ == "__main__":
    main()
