"""Build libwatersim.so (the CUDA library behind include/watersim.h) for sm_100a.

Compiles every csrc/*.cu with nvcc into one shared library in this folder.
-fmad=false: the reference computes in JavaScript doubles and never fuses a
multiply-add, so neither does the device arithmetic that mirrors it. The
learned warm start (ws_unet*.cu) has no reference arithmetic to mirror and
is built with contraction on.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libwatersim.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-fmad=false", "-Xcompiler", "-fPIC,-ffp-contract=off",
         "--expt-relaxed-constexpr"]


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def needs_build():
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(HERE, "..", "include", "watersim.h"))
    return any(os.path.getmtime(p) > t for p in deps)


def build(verbose=False, force=False, jobs=8):
    if not force and not needs_build():
        return OUT
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs, procs = [], []
    for src in sources():
        obj = os.path.join(objdir, os.path.basename(src)[:-3] + ".o")
        objs.append(obj)
        flags = FLAGS
        if os.path.basename(src).startswith("ws_unet"):
            flags = ["-fmad=true" if f == "-fmad=false" else f for f in FLAGS]
        cmd = [NVCC, *ARCH, *flags, "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd))
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
        if len(procs) >= jobs:
            _wait(procs.pop(0))
    for p in procs:
        _wait(p)
    # --no-undefined: a declaration left behind by a signature change fails here, not at load time
    link = [NVCC, *ARCH, "-shared", "-o", OUT, *objs, "-lcudart", "-Xlinker", "--no-undefined"]
    if verbose:
        print(" ".join(link))
    r = subprocess.run(link, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)
    if r.returncode:
        raise RuntimeError("link failed:\n" + r.stdout.decode())
    return OUT


def _wait(item):
    src, p = item
    out, _ = p.communicate()
    if p.returncode:
        raise RuntimeError("nvcc failed on %s:\n%s" % (src, out.decode()))


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force="-f" in sys.argv)
    print(OUT)
