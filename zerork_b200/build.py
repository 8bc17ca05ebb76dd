"""Build the sm_100a shared library in-tree: zerork_b200/lib/libzerork_b200.so.

nvcc cross-compiles for sm_100a without a GPU, so this runs on any machine
with the CUDA 12.9 toolkit.  An object file is rebuilt when its source or a
header it includes (directly or not) is newer; objects of sources that no
longer exist are not linked.
"""
import concurrent.futures as cf
import glob
import os
import re
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


_INC = re.compile(r'^\s*#\s*include\s+"([^"]+)"', re.M)


def _deps(src, seen=None):
    """The quoted includes of src, recursively (csrc/ and include/)."""
    seen = set() if seen is None else seen
    with open(src) as f:
        text = f.read()
    for name in _INC.findall(text):
        for d in (os.path.dirname(src), CSRC, os.path.join(HERE, "..", "include")):
            path = os.path.normpath(os.path.join(d, name))
            if os.path.exists(path):
                if path not in seen:
                    seen.add(path)
                    _deps(path, seen)
                break
    return seen


def _compile(src, verbose=False):
    obj = os.path.join(OBJ, os.path.basename(src) + ".o")
    newest = max([os.path.getmtime(src)] + [os.path.getmtime(h) for h in _deps(src)])
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
