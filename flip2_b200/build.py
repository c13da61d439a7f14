"""Build libflip2_b200.so in-tree for sm_100a (nvcc cross-compiles without a GPU).

The library is compiled with nvcc directly: every .cu file of csrc/ to an
object, then one shared library.  No JIT, nothing under ~/.cache: the .so sits
in flip2_b200/lib/ next to the sources.
"""
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
OBJDIR = os.path.join(LIBDIR, "obj")
LIBNAME = "libflip2_b200.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2", "--expt-relaxed-constexpr",
              "-I" + os.path.join(ROOT, "include"), "-I" + CSRC] + ARCH


def nvcc():
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(exe):
        raise RuntimeError("nvcc not found")
    return exe


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hs += [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include")) if f.endswith(".h")]
    return hs


def _compile(src, extra):
    obj = os.path.join(OBJDIR, os.path.basename(src)[:-3] + ".o")
    if _stale(obj, [src] + _headers()) or extra:
        cmd = [nvcc()] + NVCC_FLAGS + list(extra) + ["-c", src, "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed for %s:\n%s\n%s" % (src, " ".join(cmd), r.stderr[-6000:]))
        return obj, r.stderr
    return obj, ""


def build(verbose=False, extra=()):
    os.makedirs(OBJDIR, exist_ok=True)
    srcs = sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        results = list(ex.map(lambda s: _compile(s, extra), srcs))
    objs = [o for o, _ in results]
    if verbose:
        for o, log in results:
            if log:
                print(os.path.basename(o), log)
    lib = os.path.join(LIBDIR, LIBNAME)
    if _stale(lib, objs) or extra:
        cmd = [nvcc(), "-shared"] + ARCH + ["-o", lib] + objs + ["-lcurand_static", "-lculibos"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            # curand device API is header-only; link without the static host library
            cmd = [nvcc(), "-shared"] + ARCH + ["-o", lib] + objs
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError("link failed:\n" + r.stderr[-4000:])
    drv_src = os.path.join(HERE, "driver", "main.cpp")
    drv = os.path.join(LIBDIR, "flip2_main")
    if os.path.exists(drv_src) and (_stale(drv, [drv_src, lib] + _headers()) or extra):
        cmd = [nvcc(), "-O2", "-std=c++17", "-x", "cu"] + ARCH + ["-I" + os.path.join(ROOT, "include"), drv_src,
                                                                   "-o", drv, "-L" + LIBDIR, "-lflip2_b200",
                                                                   "-Xlinker", "-rpath,$ORIGIN"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("driver build failed:\n" + r.stderr[-4000:])
    return lib


if __name__ == "__main__":
    v = "-v" in sys.argv
    extra = ["-Xptxas", "-v"] if "--ptxas" in sys.argv else []
    print(build(verbose=v or bool(extra), extra=extra))
