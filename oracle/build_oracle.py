"""Build recipe for the test oracle (TEST INFRASTRUCTURE ONLY).

Outputs:
  oracle/_build/libemu_oracle.so   the C restatement (oracle/emu_oracle.c)
  oracle/_ref/libemurefinit.so     the reference's direction-set and Minerbo
                                   helpers (FlavoredNeutrinoContainerInit.cpp)
  oracle/_ref/gen<N>/Source/generated_files/*   the reference generator's output
  oracle/_ref/libemuref<N>.so      the reference's generated kernel bodies,
                                   compiled inside oracle/ref_harness.cpp

The reference tree is only read here (generator run with --emu_home pointing
into oracle/_ref, headers included from their own location).  When the
reference tree is absent (a GPU box) the prebuilt libraries are used as they
are.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF_ROOT = os.environ.get("EMU_REFERENCE_ROOT", "/root/reference")
BUILD = os.path.join(HERE, "_build")
REF_OUT = os.path.join(HERE, "_ref")

CFLAGS = ["-O2", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off"]


def _newer(out, srcs):
    if not os.path.exists(out):
        return False
    t = os.path.getmtime(out)
    return all(os.path.getmtime(s) <= t for s in srcs if os.path.exists(s))


def build_oracle(force=False):
    os.makedirs(BUILD, exist_ok=True)
    src = os.path.join(HERE, "emu_oracle.c")
    hdr = os.path.join(HERE, "emu_oracle.h")
    out = os.path.join(BUILD, "libemu_oracle.so")
    if force or not _newer(out, [src, hdr]):
        subprocess.check_call(["gcc", "-std=c99", "-D_DEFAULT_SOURCE"] + CFLAGS + [src, "-o", out, "-lm"])
    return out


def _generate(nf):
    gen_home = os.path.join(REF_OUT, "gen%d" % nf)
    fills = os.path.join(gen_home, "Source", "generated_files")
    if os.path.isdir(fills) and len(os.listdir(fills)) >= 13:
        return gen_home
    os.makedirs(gen_home, exist_ok=True)
    script_dir = os.path.join(REF_ROOT, "Scripts", "symbolic_hermitians")
    subprocess.check_call([sys.executable, os.path.join(script_dir, "generate_code.py"), str(nf),
                           "--emu_home", gen_home], cwd=script_dir,
                          stdout=subprocess.DEVNULL)
    return gen_home


def build_ref(force=False):
    """Build oracle/_ref/libemuref{2,3}.so; returns the list of libraries (may
    be empty when neither the reference tree nor prebuilt outputs exist)."""
    outs = []
    have_ref = os.path.isdir(os.path.join(REF_ROOT, "Source"))
    for nf in (2, 3):
        out = os.path.join(REF_OUT, "libemuref%d.so" % nf)
        if not have_ref:
            if os.path.exists(out):
                outs.append(out)
            continue
        gen_home = _generate(nf)
        src = os.path.join(HERE, "ref_harness.cpp")
        deps = [src, os.path.join(HERE, "emu_oracle.h"), os.path.join(HERE, "shim", "AMReX_REAL.H")]
        if force or not _newer(out, deps):
            cmd = ["g++", "-std=c++17"] + CFLAGS + [
                "-I", os.path.join(HERE, "shim"),
                "-I", HERE,
                "-I", os.path.join(REF_ROOT, "Source"),
                "-I", os.path.join(gen_home, "Source"),
                src, "-o", out]
            subprocess.check_call(cmd)
        outs.append(out)
    return outs


def build_ref_init(force=False):
    """oracle/_ref/libemurefinit.so: the helper functions at the top of the
    reference's Source/FlavoredNeutrinoContainerInit.cpp (every line before
    the FlavoredNeutrinoContainer constructor: uniform_sphere_xyz,
    minerbo_Z, minerbo_closure, ...), unmodified except that their two
    #include lines give way to oracle/shim/ref_init_shim.h, followed by
    oracle/ref_init_api.inc.  None when neither the reference tree nor a
    prebuilt library exists."""
    out = os.path.join(REF_OUT, "libemurefinit.so")
    src = os.path.join(REF_ROOT, "Source", "FlavoredNeutrinoContainerInit.cpp")
    if not os.path.exists(src):
        return out if os.path.exists(out) else None
    api = os.path.join(HERE, "ref_init_api.inc")
    shim = os.path.join(HERE, "shim", "ref_init_shim.h")
    if not force and _newer(out, [src, api, shim]):
        return out
    lines = open(src).read().splitlines()
    end = next(i for i, l in enumerate(lines) if l.startswith("FlavoredNeutrinoContainer::"))
    body = ["// (shim) " + l if l.lstrip().startswith("#include \"") else l for l in lines[:end]]
    os.makedirs(REF_OUT, exist_ok=True)
    tu = os.path.join(REF_OUT, "ref_init_tu.cpp")
    with open(tu, "w") as f:
        f.write('#include "ref_init_shim.h"\n')
        f.write('#line 1 "%s"\n' % src)
        f.write("\n".join(body) + "\n")
        f.write('#include "ref_init_api.inc"\n')
    subprocess.check_call(["g++", "-std=c++17"] + CFLAGS + ["-I", os.path.join(HERE, "shim"), "-I", HERE, tu,
                           "-o", out])
    return out


def build_all(force=False):
    a = build_oracle(force)
    b = build_ref(force)
    c = build_ref_init(force)
    return [a] + b + ([c] if c else [])


if __name__ == "__main__":
    for p in build_all(force="--force" in sys.argv):
        print(p)
