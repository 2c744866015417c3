"""Build recipe for the native libraries of this repository.

lib/libpixgpu.so    the B200 chain (CUDA, sm_100a) behind include/pixgpu.h
lib/libpixsynth.so  the seeded synthetic detector/event generator (include/pixsynth.h)
lib/pluginPixelB200.so  the chain's modules for the reference framework (framework/), built
                    against that framework's headers (only where the reference tree exists)
oracle/liboracle.so the CPU oracle used by the tests (checker only)
oracle/_ref/        checker build of the reference's serial sources (only where they exist)

Everything is compiled in-tree so the libraries travel with the repository.
"""
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
LIB = os.path.join(PKG, "lib")
CSRC = os.path.join(PKG, "csrc")
INC = os.path.join(ROOT, "include")
OBJ = os.path.join(PKG, "_build")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# --fmad=false: the reference's serial arithmetic has no fused multiply-add,
# and bit-exact cluster/hit/doublet/tuple results depend on it.
NVFLAGS = ["-O3", "-std=c++17", "-lineinfo", "--fmad=false", "-Xcompiler", "-fPIC", "-I", INC, "-I", CSRC,
           "--expt-relaxed-constexpr"] + ARCH
CU_SOURCES = ["scan.cu", "k_local.cu", "k_ca.cu", "k_fit.cu", "k_vertex.cu", "k_pack.cu", "chain.cu", "capi.cu",
              "pool.cu", "serve.cu", "noalloc.cu", "fedscan.cu", "tune.cu"]


def _run(cmd):
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        raise RuntimeError("build step failed: %s\n%s" % (" ".join(cmd), r.stdout))
    return r.stdout


def _stale(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def _headers(d):
    return [os.path.join(d, f) for f in os.listdir(d) if f.endswith((".h", ".cuh"))]


def build_gpu(verbose=False):
    os.makedirs(LIB, exist_ok=True)
    os.makedirs(OBJ, exist_ok=True)
    target = os.path.join(LIB, "libpixgpu.so")
    deps = _headers(CSRC) + _headers(INC)
    objs, jobs = [], []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src + ".o")
        objs.append(o)
        if _stale(o, [s] + deps):
            jobs.append([NVCC] + NVFLAGS + ["-c", s, "-o", o])
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        for out in ex.map(_run, jobs):
            if verbose and out.strip():
                print(out)
    if jobs or _stale(target, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", target] + objs + ["-lcudart"])
    return target


def build_synth():
    os.makedirs(LIB, exist_ok=True)
    src = os.path.join(CSRC, "synth", "pixsynth.cc")
    target = os.path.join(LIB, "libpixsynth.so")
    if _stale(target, [src] + _headers(INC)):
        _run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-I", INC, src, "-o", target])
    return target


def build_oracle():
    d = os.path.join(ROOT, "oracle")
    srcs = [os.path.join(d, f) for f in ("oracle_local.cc", "oracle_ca.cc", "oracle_fit.cc", "oracle_riemann.cc",
                                         "oracle_vertex.cc", "oracle_api.cc")]
    target = os.path.join(d, "liboracle.so")
    if _stale(target, srcs + [os.path.join(d, h) for h in ("oracle.h", "oracle_mat.h", "sym_eigen.h")] + _headers(INC)):
        _run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-pthread", "-I", INC] + srcs + ["-o", target])
    return target


def reference_dir():
    """The reference checkout the checker builds read: $PIXTRACK_REFERENCE, else
    the container's read-only mount.  None where neither exists (the GPU box)."""
    for d in (os.environ.get("PIXTRACK_REFERENCE"), "/root/reference"):
        if d and os.path.isdir(os.path.join(d, "src", "serial")):
            return d
    return None


def build_plugins(reference=None):
    """The framework modules (framework/Makefile), against the reference framework's headers."""
    reference = reference or reference_dir()
    if reference is None:
        return None
    _run(["make", "-s", "-j8", "-C", os.path.join(PKG, "framework"), "REF=" + reference])
    return os.path.join(LIB, "pluginPixelB200.so")


def build_ref(reference=None):
    """Checker build of the reference serial sources and of its event processor with
    the plugins (skipped where the reference tree is absent)."""
    reference = reference or reference_dir()
    if reference is None:
        return None
    _run(["make", "-s", "-j8", "-C", os.path.join(ROOT, "oracle", "ref"), "REF=" + reference])
    if os.path.exists(os.path.join(LIB, "pluginPixelB200.so")):
        _run(["make", "-s", "-j8", "-C", os.path.join(ROOT, "oracle", "ref"), "REF=" + reference, "fw"])
    return os.path.join(ROOT, "oracle", "_ref", "libpixref.so")


def build_all(gpu=True):
    out = {"synth": build_synth(), "oracle": build_oracle()}
    if gpu:
        out["gpu"] = build_gpu()
        out["plugins"] = build_plugins()
    out["ref"] = build_ref()
    return out


if __name__ == "__main__":
    print(build_all(gpu="--no-gpu" not in sys.argv))
