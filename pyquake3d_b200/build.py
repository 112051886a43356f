"""Build libpq3d.so in-tree with nvcc for sm_100a.

The library is built next to this file so it travels with the source tree;
the product never falls back to anything else when it is missing.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libpq3d.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
SOURCES = ["gf.cu", "aca.cu", "hmatvec.cu", "mixed_pack.cu", "rk.cu", "ensemble.cu", "vmode.cu", "mlp.cu", "hostio.cu"]
EXTRA = {}
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
    "-cudart", "static",
]


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def needs_build():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    for f in os.listdir(CSRC):
        if os.path.getmtime(os.path.join(CSRC, f)) > t:
            return True
    return False


def build(force=False, verbose=False):
    if not force and not needs_build():
        return LIB
    import tempfile
    from concurrent.futures import ThreadPoolExecutor
    tmp = tempfile.mkdtemp(prefix="pq3d_build_")
    objs = []
    cmds = []
    for s in SOURCES:
        o = os.path.join(tmp, s + ".o")
        objs.append(o)
        cmds.append([_nvcc()] + NVCC_FLAGS + EXTRA.get(s, []) + ["-I", CSRC, "-I", INCLUDE, "-c",
                                                                   os.path.join(CSRC, s), "-o", o])
    with ThreadPoolExecutor(len(cmds)) as ex:
        for c in cmds:
            if verbose:
                print(" ".join(c))
        list(ex.map(lambda c: subprocess.run(c, check=True), cmds))
    link = [_nvcc(), "-shared", "-cudart", "static", "-gencode", "arch=compute_100a,code=sm_100a",
            "-o", LIB + ".tmp"] + objs
    subprocess.run(link, check=True)
    os.replace(LIB + ".tmp", LIB)
    for o in objs:
        os.remove(o)
    os.rmdir(tmp)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
