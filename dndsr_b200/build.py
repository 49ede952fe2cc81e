"""Builds the CUDA library dndsr_b200/libdndsb.so for sm_100a with nvcc."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = ["setup.cu", "hotpath.cu", "fast.cu", "reduce.cu", "linsolve.cu", "bc.cu", "adjoint.cu", "adjoint_roe.cu", "adjoint_fast.cu", "adjoint_fast_sa.cu", "adjoint_visc.cu", "adjoint_ops.cu", "adjoint_geom.cu", "adjoint_geom2d.cu", "adjoint_generic.cu", "adjoint_generic_p1n5.cu", "adjoint_generic_p1n6.cu", "adjoint_generic_p2n5.cu", "adjoint_generic_p2n6.cu", "positivity.cu", "limiter.cu", "capi.cu", "noalloc.cu", "roejac.cu"]
LIB = os.path.join(HERE, "libdndsb.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
         "--expt-relaxed-constexpr", "-ccbin", "/usr/bin/g++"]


def sources():
    d = os.path.join(HERE, "csrc")
    return [os.path.join(d, s) for s in SRC]


def _deps():
    d = os.path.join(HERE, "csrc")
    inc = os.path.join(os.path.dirname(HERE), "include")
    return [os.path.join(d, f) for f in os.listdir(d)] + [os.path.join(inc, f) for f in os.listdir(inc)]


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(p) <= t for p in _deps())


def _includes_mtime(path, seen=None):
    """Newest modification time of a source and of the local headers it includes, recursively."""
    import re
    seen = set() if seen is None else seen
    if path in seen or not os.path.exists(path):
        return 0.0
    seen.add(path)
    t = os.path.getmtime(path)
    base = os.path.dirname(path)
    with open(path) as fh:
        for name in re.findall(r'^\s*#\s*include\s+"([^"]+)"', fh.read(), flags=re.M):
            t = max(t, _includes_mtime(os.path.normpath(os.path.join(base, name)), seen))
    return t


def _ext_path():
    import sysconfig
    return os.path.join(HERE, "_C" + sysconfig.get_config_var("EXT_SUFFIX"))


def build_pybind(force=False):
    """The pybind11 module dndsr_b200/_C (host C++ over the C-ABI), linked to libdndsb.so by an $ORIGIN rpath."""
    import sysconfig
    import pybind11
    src = os.path.join(HERE, "csrc", "pybind.cpp")
    out = _ext_path()
    hdr = os.path.join(os.path.dirname(HERE), "include", "dndsb.h")
    if not force and os.path.exists(out) and os.path.getmtime(out) >= max(os.path.getmtime(src), os.path.getmtime(hdr), os.path.getmtime(LIB)):
        return out
    cmd = ["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-fvisibility=hidden", "-I", pybind11.get_include(), "-I",
           sysconfig.get_paths()["include"], src, "-o", out, "-L", HERE, "-ldndsb", "-Wl,-rpath,$ORIGIN"]
    subprocess.check_call(cmd)
    return out


def build(force=False, verbose=False, jobs=None):
    if not force and up_to_date():
        build_pybind()
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    procs = []
    for s in sources():
        o = os.path.join(objdir, os.path.basename(s) + ".o")
        objs.append(o)
        # an object is reused when it is newer than its source and every local header the source includes
        if not force and not verbose and os.path.exists(o) and os.path.getmtime(o) >= _includes_mtime(s):
            continue
        cmd = [NVCC, *FLAGS, "-c", s, "-o", o]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
            print(" ".join(cmd), flush=True)
        procs.append((s, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    failed = False
    for s, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0 or verbose:
            sys.stdout.write(out.decode(errors="replace"))
        failed |= p.returncode != 0
    if failed:
        raise RuntimeError("nvcc failed")
    subprocess.check_call([NVCC, *FLAGS, "-shared", "-o", LIB, *objs, "-lcudart"])
    build_pybind(force=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
