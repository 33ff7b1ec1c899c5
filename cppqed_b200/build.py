"""Builds the engine library ``cppqed_b200/_lib/libcqg.so`` for sm_100a.

The host sources (element library, model builder, lowering, errors) are compiled
with g++, the CUDA sources with nvcc (``-gencode arch=compute_100a,code=sm_100a``),
and everything is linked into one shared library exporting the C ABI of
``include/cqg.h`` and ``include/cqg_model.h``.  Rebuilds only what is out of date.
"""
import hashlib
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "_lib")
OBJDIR = os.path.join(HERE, "_build")
LIB = os.path.join(LIBDIR, "libcqg.so")

HOST_SOURCES = ["host/tridiagonal.cpp", "host/elements.cpp", "host/model.cpp", "host/pars.cpp",
                "host/scripts.cpp", "host/errors.cpp", "host/api_model.cpp", "host/lowering.cpp"]
CUDA_SOURCES = ["cuda/api.cu", "cuda/noalloc.cu", "cuda/kernels_block.cu", "cuda/apply.cu", "cuda/server.cu", "cuda/master.cu"]
# the kernel instantiations: one object per (precision, rows per lane)
KERNEL_INSTANCES = [(r, e, ip) for r in ("double", "float") for e in (1, 2, 3, 4) for ip in (0, 1)]
# what each kind of object is rebuilt for (besides its own source and include/*.h)
HOST_HEADERS = ["host/lowering.hpp", "host/errors.hpp", "host/model.hpp", "host/elements.hpp", "host/tridiagonal.hpp",
                "host/pars.hpp"]
KERNEL_HEADERS = ["cuda/mcwf_kernel.cuh", "cuda/rng.cuh"]
CUDA_HEADERS = ["cuda/engine_internal.cuh", "cuda/mcwf_kernel.cuh", "cuda/mcwf_block.cuh", "cuda/rng.cuh",
                "host/lowering.hpp", "host/errors.hpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc():
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _digest(files, cmd):
    """Content hash of an object's inputs and its command line."""
    h = hashlib.sha256(" ".join(cmd).encode())
    for f in files:
        with open(f, "rb") as fh:
            h.update(fh.read())
    return h.hexdigest()


def _needs_compile(obj, files, cmd):
    """An object is rebuilt unless its stamp holds the hash of the inputs it was compiled
    from.  The hash is taken before the compiler starts, so a source edited while it compiles
    leaves a stamp that no longer matches."""
    d = _digest(files, cmd)
    try:
        with open(obj + ".stamp") as fh:
            ok = os.path.exists(obj) and fh.read() == d
    except OSError:
        ok = False
    return (not ok), d


def _stamp(obj, d):
    with open(obj + ".stamp", "w") as fh:
        fh.write(d)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("build step failed: " + " ".join(cmd[:3]) + " ...")
    return r.stdout + r.stderr


def build(verbose=False, ptxas_info=False, extra_flags=(), lib=None):
    os.makedirs(LIBDIR, exist_ok=True)
    os.makedirs(OBJDIR, exist_ok=True)
    inc = ["-I" + os.path.join(ROOT, "include")]
    public = [os.path.join(ROOT, "include", h) for h in ("cqg.h", "cqg_model.h")]

    def deps(names, with_public=True):
        return [os.path.join(CSRC, h) for h in names] + (public if with_public else [])

    objs = []
    for src in HOST_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJDIR, os.path.basename(src) + ".o")
        cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-Wall", *inc, "-c", s, "-o", o]
        need, d = _needs_compile(o, [s] + deps(HOST_HEADERS), cmd)
        if need:
            _run(cmd, verbose)
            _stamp(o, d)
        objs.append(o)
    info = ""
    jobs = []
    for src in CUDA_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJDIR, os.path.basename(src) + ".o")
        jobs.append((s, o, [], deps(CUDA_HEADERS)))
    inst = os.path.join(CSRC, "cuda", "kernels_inst.cu")
    for r, e, ip in KERNEL_INSTANCES:
        jobs.append((inst, os.path.join(OBJDIR, "kernels_%s_e%d_ip%d.o" % (r, e, ip)),
                     ["-DCQG_REAL=" + r, "-DCQG_E=%d" % e, "-DCQG_IP=%d" % ip],
                     deps(KERNEL_HEADERS, with_public=False)))
    procs = []
    for s, o, defs, hdrs in jobs:
        objs.append(o)
        cmd = [_nvcc(), *ARCH, "-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", *inc, *defs,
               *extra_flags, "-c", s, "-o", o]
        need, d = _needs_compile(o, [s] + hdrs, cmd)
        if need or ptxas_info:
            if ptxas_info:
                cmd.insert(1, "-Xptxas=-v")
            if verbose:
                print(" ".join(cmd), flush=True)
            procs.append((cmd, o, d, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT,
                                                     text=True)))
    for cmd, o, d, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            sys.stderr.write(out)
            raise RuntimeError("build step failed: " + " ".join(cmd[:3]) + " ...")
        _stamp(o, d)
        info += out
    out = lib or LIB
    if _stale(out, objs):
        _run([_nvcc(), *ARCH, "-shared", "-o", out, *objs, "-lcudart"], verbose)
    if lib is None:
        build_apps(verbose)
    return info


APPS = {"cqg_evolve": "apps/cqg_evolve.cpp"}


def build_apps(verbose=False):
    """The C++ programs over the C ABI (include/cqg_ensemble.hpp), linked against libcqg.so
    in the same directory."""
    inc = os.path.join(ROOT, "include")
    for name, src in APPS.items():
        s = os.path.join(CSRC, src)
        exe = os.path.join(LIBDIR, name)
        deps = [s, LIB] + [os.path.join(inc, h) for h in ("cqg.h", "cqg_model.h", "cqg_ensemble.hpp")]
        if _stale(exe, deps):
            _run(["g++", "-std=c++17", "-O2", "-Wall", "-I" + inc, s, "-L" + LIBDIR, "-lcqg",
                  "-Wl,-rpath,$ORIGIN", "-o", exe], verbose)


if __name__ == "__main__":
    txt = build(verbose=True, ptxas_info="--ptxas-info" in sys.argv)
    if txt:
        print(txt)
