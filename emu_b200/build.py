"""Build the CUDA library libemu_b200.so in-tree (sm_100a) and the host
driver emu_main that runs the reference's inputs files through it.

    python -m emu_b200.build [--force] [--verbose-ptxas]

Objects go to emu_b200/_build/, the shared library to emu_b200/libemu_b200.so
and the driver to emu_b200/emu_main (next to this file, so both travel with
the source tree).  nvcc cross-compiles without a GPU.
"""
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libemu_b200.so")
MAIN = os.path.join(HERE, "emu_main")
INCLUDE = os.path.join(ROOT, "include")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I", INCLUDE, "-I", CSRC]

SOURCES = ["emu_k_fp64_3.cu", "emu_k_mixed_3.cu", "emu_adjoint.cu", "emu_k_fp64_2.cu", "emu_k_mixed_2.cu",
           "emu_k_misc.cu", "emu_capi.cu", "emu_comm.cu", "emu_noalloc.cu", "emu_init_device.cu", "emu_host.cpp",
           "emu_init.cpp"]
# the device initial-condition generator must round like the host one
EXTRA = {"emu_init_device.cu": ["-fmad=false"]}
HEADERS = ["emu_device.cuh", "emu_kernels.cuh", "emu_kernels_impl.cuh", "emu_context.cuh", "emu_host.h",
           "emu_init_record.h"]


def _stale(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src, verbose_ptxas):
    path = os.path.join(CSRC, src)
    obj = os.path.join(OBJ, src + ".o")
    deps = [path] + [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "emu_b200.h")]
    if not _stale(obj, deps):
        return obj, ""
    cmd = [NVCC] + ARCH + COMMON + EXTRA.get(src, []) + ["-c", path, "-o", obj]
    if src.endswith(".cu"):
        cmd += ["--extended-lambda", "-Xptxas", "-warn-spills"]
        if verbose_ptxas:
            cmd += ["-Xptxas", "-v"]
    else:
        cmd += ["-x", "c++"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed for %s:\n%s\n%s" % (src, r.stdout, r.stderr))
    return obj, r.stderr


def build(force=False, verbose_ptxas=False, quiet=True):
    os.makedirs(OBJ, exist_ok=True)
    if force:
        for s in SOURCES:
            o = os.path.join(OBJ, s + ".o")
            if os.path.exists(o):
                os.remove(o)
    with cf.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        results = list(ex.map(lambda s: _compile(s, verbose_ptxas), SOURCES))
    objs = [r[0] for r in results]
    logs = "".join(r[1] for r in results)
    if logs and not quiet:
        sys.stderr.write(logs)
    if force or _stale(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart", "-ldl"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n%s\n%s" % (r.stdout, r.stderr))
    main_src = os.path.join(CSRC, "emu_main.cpp")
    if force or _stale(MAIN, [main_src, LIB, os.path.join(INCLUDE, "emu_b200.h")]):
        cmd = ["g++", "-O2", "-std=c++17", "-I", INCLUDE, main_src, "-o", MAIN, "-L", HERE, "-lemu_b200",
               "-Wl,-rpath,$ORIGIN"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("emu_main build failed:\n%s\n%s" % (r.stdout, r.stderr))
    return LIB, logs


if __name__ == "__main__":
    lib, logs = build(force="--force" in sys.argv, verbose_ptxas="--verbose-ptxas" in sys.argv, quiet=False)
    print(lib)
