"""Build the galfast_b200 native library for sm_100a.

    python -m galfast_b200.build          # or galfast_b200.build.build()

compiles every CUDA and C++ source under galfast_b200/csrc (one nvcc process
per source file, in parallel) into galfast_b200/_lib/libgalfast_b200.so and writes the stream-multiplier table
(safeprimes_65536.bin) next to it.  Device code is compiled with -fmad=false
and host code with -ffp-contract=off: the catalog's Poisson draws depend on the
exact float results of the reference's expressions, so no multiply-add may be
fused unless the source asks for it (gf_math.h uses explicit fma).
"""
import ctypes
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "_lib")
LIBNAME = "libgalfast_b200.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

SOURCES = ["gf_skygen.cu", "gf_modules.cu", "gf_api.cu", "gf_static.cu", "gf_multi.cu", "gf_integrate.cu", "gf_batchdraw.cu", "gf_precision.cu", "gf_server.cpp", "gf_host.cpp", "gf_safeprimes.cpp", "gf_textout.cpp"]


def nvcc_path():
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found")
    return cand


def _flags(extra):
    return [*ARCH, "-O3", "-lineinfo", "-std=c++17", "-fmad=false", "--expt-relaxed-constexpr",
            "-Xcompiler", "-fPIC,-ffp-contract=off,-fno-fast-math", *(extra or [])]


def build(verbose=False, extra=None, jobs=None):
    """Compile every source to an object file (in parallel), then link the shared
    library.  No device symbol crosses a source file, so no device link is needed."""
    from concurrent.futures import ThreadPoolExecutor
    os.makedirs(LIBDIR, exist_ok=True)
    objdir = os.path.join(LIBDIR, "obj")
    os.makedirs(objdir, exist_ok=True)
    out = os.path.join(LIBDIR, LIBNAME)
    nvcc = nvcc_path()

    def compile_one(src):
        obj = os.path.join(objdir, os.path.splitext(src)[0] + ".o")
        cmd = [nvcc, *_flags(extra), "-c", "-o", obj, os.path.join(CSRC, src)]
        if verbose:
            print(" ".join(cmd))
        r = subprocess.run(cmd, capture_output=True, text=True)
        return obj, r

    n = jobs or min(len(SOURCES), os.cpu_count() or 1)
    with ThreadPoolExecutor(max_workers=n) as ex:
        results = list(ex.map(compile_one, SOURCES))
    for (obj, r), src in zip(results, SOURCES):
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("nvcc build of %s failed (%s)" % (LIBNAME, src))
    cmd = [nvcc, *ARCH, "-shared", "-o", out, *[o for o, _ in results], "-ldl", "-lpthread"]
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("link of %s failed" % LIBNAME)
    write_multiplier_table(out)
    return out


def write_multiplier_table(libpath):
    """Regenerate the 65536 stream multipliers (primality tests, ~5 s) once."""
    fn = os.path.join(LIBDIR, "safeprimes_65536.bin")
    if os.path.exists(fn) and os.path.getsize(fn) == 65536 * 4:
        return fn
    lib = ctypes.CDLL(libpath)
    buf = (ctypes.c_uint32 * 65536)()
    if lib.gf_multipliers(buf, 65536) != 0:
        raise RuntimeError("multiplier generation failed")
    with open(fn, "wb") as f:
        f.write(bytes(buf))
    return fn


if __name__ == "__main__":
    print(build(verbose=True))
