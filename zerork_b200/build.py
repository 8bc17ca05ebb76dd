"""Build the sm_100a shared library in-tree: zerork_b200/lib/libzerork_b200.so.

nvcc cross-compiles for sm_100a without a GPU, so this runs on any machine
with the CUDA 12.9 toolkit.  Object files are rebuilt when their source or any
header in csrc/ is newer.
"""
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB_DIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIB_DIR, "libzerork_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    for c in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _flags(src):
    common = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O3",
              f"-I{CSRC}", f"-I{os.path.join(HERE, '..', 'include')}"]
    if src.endswith(".cu"):
        return ARCH + common + ["--expt-relaxed-constexpr", "-Xptxas", "-O3"]
    return ARCH + common


def _compile(src, verbose=False):
    obj = os.path.join(OBJ, os.path.basename(src) + ".o")
    headers = (glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) +
               glob.glob(os.path.join(HERE, "..", "include", "*.h")))
    newest = max([os.path.getmtime(src)] + [os.path.getmtime(h) for h in headers])
    if os.path.exists(obj) and os.path.getmtime(obj) >= newest:
        return obj, None
    cmd = [nvcc(), "-c", src, "-o", obj] + _flags(src)
    if verbose and src.endswith(".cu"):
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    # date the object by the inputs it was compiled from, so that a source
    # edited while the compiler ran counts as newer on the next build
    os.utime(obj, (newest, newest))
    return obj, r.stderr


def build(verbose=False):
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(LIB_DIR, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        res = list(ex.map(lambda s: _compile(s, verbose), srcs))
    objs = [o for o, _ in res]
    if verbose:
        for _, log in res:
            if log:
                print(log)
    compiled = any(log is not None for _, log in res)
    if compiled or not os.path.exists(LIB):
        cmd = [nvcc(), "-shared", "-o", LIB] + ARCH + objs + ["-lcudart_static", "-ldl", "-lrt", "-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
