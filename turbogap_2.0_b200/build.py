"""Build libtgap.so (CUDA kernels + C ABI) for sm_100a, in-tree.

    python turbogap_2.0_b200/build.py [--force] [--verbose]

Objects go to turbogap_2.0_b200/_build/, the library to turbogap_2.0_b200/lib/libtgap.so.
Each translation unit is rebuilt when it or any header of csrc/ changed.
"""
import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libtgap.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

# (source, extra flags). The neighbor builder must not contract multiply-adds: the accept
# test d < rcut has to see the bits of the reference arithmetic.
SOURCES = [
    ("capi.cu", []),
    ("neighbors.cu", ["--fmad=false"]),
    ("soap.cu", []),
    ("soap_fwd_f32.cu", []),
    ("soap_fwd_f64.cu", []),
    ("soap_bwd_f32.cu", []),
    ("soap_bwd_f64.cu", []),
    ("soap_fwd_f32_cmp.cu", []),
    ("soap_fwd_f64_cmp.cu", []),
    ("soap_bwd_f32_cmp.cu", []),
    ("soap_bwd_f64_cmp.cu", []),
    ("gap.cu", []),
    ("gemm_tc.cu", []),
    ("md.cu", []),
    ("mc.cu", ["--fmad=false"]),
    ("screen.cu", []),
    ("screen_train.cu", []),
    ("pair_terms.cu", []),
    ("tables.cpp", []),
]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def host_cxx():
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"


def _headers_mtime():
    m = 0.0
    for d in (CSRC, os.path.join(ROOT, "include")):
        for f in os.listdir(d):
            if f.endswith((".h", ".cuh", ".hpp")):
                m = max(m, os.path.getmtime(os.path.join(d, f)))
    return m


def _compile(src, extra, force, verbose):
    s = os.path.join(CSRC, src)
    o = os.path.join(OBJ, src + ".o")
    if not force and os.path.exists(o) and os.path.getmtime(o) >= max(os.path.getmtime(s), _headers_mtime()):
        return o
    if src.endswith(".cpp"):
        cmd = [host_cxx(), "-O2", "-fPIC", "-std=gnu++17", "-ffp-contract=off",
               "-I/usr/local/cuda/include", "-c", s, "-o", o]
    else:
        cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
               "-ccbin", host_cxx(), "-Xptxas", "-warn-spills", *extra, "-c", s, "-o", o]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {src}\n{r.stdout}\n{r.stderr}")
    if verbose and (r.stdout or r.stderr):
        print(r.stdout, r.stderr)
    return o


def build(force=False, verbose=False):
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 2)) as ex:
        objs = list(ex.map(lambda a: _compile(a[0], a[1], force, verbose), SOURCES))
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= max(os.path.getmtime(o) for o in objs):
        return LIB
    cmd = [nvcc(), *ARCH, "-shared", "-ccbin", host_cxx(), "-o", LIB, *objs, "-cudart", "static"]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    try:
        print(build(a.force, a.verbose))
    except RuntimeError as e:
        print(e, file=sys.stderr)
        sys.exit(1)
