"""Build recipe for the B200 string sort.

Produces, in place:
  string-sorting_b200/libssort_b200.so      CUDA kernels + C ABI (sm_100a)
  string-sorting_b200/libssort_workloads.so synthetic input generators
  oracle/liboracle.so                       the test-only C oracle
  oracle/_ref/{libref.so,unit-test,sortstring}
                                            the reference compiled from its
                                            sources (only when they are present)

Run as `python string-sorting_b200/build.py` or through __graft_entry__.build().
"""
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
ORACLE = os.path.join(ROOT, "oracle")
# The reference checkout: $SSORT_REF_DIR, else a sibling directory of this
# repository named `reference`.  Without it the reference-built checkers are
# skipped (the GPU box only uses the files built beforehand).
REF_DIR = os.environ.get("SSORT_REF_DIR") or os.path.join(os.path.dirname(ROOT), "reference")

LIB = os.path.join(PKG, "libssort_b200.so")
WLIB = os.path.join(PKG, "libssort_workloads.so")
CLI = os.path.join(PKG, "ssort-sort")

GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _host_cxx():
    # The system g++ has the OpenMP spec files; an environment CXX may not.
    for c in ("/usr/bin/g++", shutil.which("g++") or ""):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("no g++ found")


def _host_cc():
    for c in ("/usr/bin/gcc", shutil.which("gcc") or ""):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("no gcc found")


def _newer(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def _run(cmd, cwd=None):
    r = subprocess.run(cmd, cwd=cwd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout)
        raise RuntimeError("build step failed: " + " ".join(cmd))
    return r.stdout


def build_cuda(force=False, extra_flags=()):
    srcs = [os.path.join(CSRC, f) for f in ("ssort_kernels.cu", "ssort_engine.cu",
                                             "ssort_graph.cu", "ssort_server.cu",
                                             "ssort_merge.cpp")]
    deps = srcs + [os.path.join(CSRC, h) for h in ("ssort_internal.cuh", "ssort_host.cuh")]
    deps.append(os.path.join(INCLUDE, "ssort_b200.h"))
    if not force and not _newer(LIB, deps):
        return LIB
    nvcc = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    tmp = LIB + ".tmp"
    cmd = [nvcc, *GENCODE, "-lineinfo", "-O3", "-std=c++17", "-shared",
           "-ccbin", _host_cxx(), "-Xcompiler", "-fPIC,-fopenmp,-O3",
           "-I", INCLUDE, "-I", CSRC, *extra_flags, *srcs, "-o", tmp, "-lgomp"]
    _run(cmd)
    os.replace(tmp, LIB)
    return LIB


def build_workloads(force=False):
    src = os.path.join(PKG, "workloads", "ssort_workloads.cpp")
    if not force and not _newer(WLIB, [src]):
        return WLIB
    tmp = WLIB + ".tmp"
    _run([_host_cxx(), "-O3", "-std=c++17", "-fPIC", "-shared", "-fopenmp", src, "-o", tmp])
    os.replace(tmp, WLIB)
    return WLIB


def build_oracle(force=False):
    make = shutil.which("make")
    env_cmd = [make, "-C", ORACLE, "CC=" + _host_cc(), "CXX=" + _host_cxx()]
    if force:
        _run(env_cmd + ["-B", "oracle"])
    else:
        _run(env_cmd + ["oracle"])
    if os.path.isdir(os.path.join(REF_DIR, "src")):
        _run(env_cmd + ["-j8", "REF_DIR=" + REF_DIR, "ref", "ref-bins"])


def build_cli(force=False):
    """ssort-sort: the whole-file command-line front end (links the library)."""
    src = os.path.join(PKG, "cli", "ssort_cli.cpp")
    if not force and not _newer(CLI, [src, LIB, os.path.join(INCLUDE, "ssort_b200.h")]):
        return CLI
    tmp = CLI + ".tmp"
    _run([_host_cxx(), "-O2", "-std=c++17", "-I", INCLUDE, src, "-o", tmp, "-L", PKG,
          "-lssort_b200", "-Wl,-rpath,$ORIGIN"])
    os.replace(tmp, CLI)
    return CLI


def build_all(force=False):
    build_cuda(force)
    build_workloads(force)
    build_cli(force)
    build_oracle(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
    print("built:", LIB, WLIB)
