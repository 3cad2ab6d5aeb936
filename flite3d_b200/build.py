"""Build the native libraries in-tree.

* ``flite3d_b200/libflite_gpu.so``    -- CUDA sm_100a solver + C ABI (nvcc)
* ``flite3d_b200/libflite_prepro.so`` -- host preprocessor and file formats
* ``oracle/_build/liboracle.so``      -- CPU restatement (test checker)

Every library is built from source with explicit compiler invocations; the
FP64 kernels and the oracle are compiled without floating-point contraction
(``--fmad=false`` / ``-ffp-contract=off``) so that their results can be
compared bit for bit.
"""
import os
import shutil
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "flite3d_b200")
INC = os.path.join(ROOT, "include")
CSRC = os.path.join(PKG, "csrc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc():
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _run(cmd, verbose=False):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd[:3])} ...")
    return r


def _stale(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def _sources(dirname, exts):
    out = []
    for base, _, files in os.walk(dirname):
        for f in sorted(files):
            if os.path.splitext(f)[1] in exts:
                out.append(os.path.join(base, f))
    return out


def build_prepro(force=False, verbose=False):
    # the controls defaults are compiled in as fp_controls_default/derive
    src = [os.path.join(CSRC, "prepro", f) for f in ("prepro.cpp", "domains.cpp", "namelist.cpp", "text_io.cpp")] + \
        [os.path.join(CSRC, "solver", "controls.cpp")]
    deps = src + _sources(os.path.join(CSRC, "prepro"), {".hpp", ".h"}) + _sources(INC, {".h"})
    out = os.path.join(PKG, "libflite_prepro.so")
    if force or _stale(out, deps):
        _run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-pthread", "-DFLITE_CONTROLS_FP", f"-I{INC}",
              *src, "-o", out], verbose)
    return out


def build_gpu(force=False, verbose=False):
    sdir = os.path.join(CSRC, "solver")
    cu = _sources(sdir, {".cu"})
    cpp = _sources(sdir, {".cpp"})
    deps = cu + cpp + _sources(sdir, {".cuh", ".h", ".hpp"}) + _sources(INC, {".h"})
    out = os.path.join(PKG, "libflite_gpu.so")
    if not (force or _stale(out, deps)):
        return out
    objdir = os.path.join(ROOT, "_build", "gpu")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    for s in cu + cpp:
        o = os.path.join(objdir, os.path.basename(s) + ".o")
        cmd = [_nvcc(), "-c", s, "-o", o, "-std=c++17", "-O3", *ARCH, "-lineinfo", "--fmad=false",
               "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off", f"-I{INC}",
               f"-I{sdir}", "--expt-relaxed-constexpr"]
        objs.append(o)
        _run(cmd, verbose)
    _run([_nvcc(), "-shared", *ARCH, "-o", out, *objs, "-cudart", "static"], verbose)
    return out


def build_oracle(force=False, verbose=False):
    odir = os.path.join(ROOT, "oracle")
    src = [os.path.join(odir, "oracle.cpp")]
    sdir = os.path.join(ROOT, "flite3d_b200", "csrc", "solver")
    deps = src + [os.path.join(odir, "oracle.h"), os.path.join(sdir, "pinned_math.h")] + _sources(INC, {".h"})
    outdir = os.path.join(odir, "_build")
    os.makedirs(outdir, exist_ok=True)
    out = os.path.join(outdir, "liboracle.so")
    if force or _stale(out, deps):
        _run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off",
              "-fno-fast-math", f"-I{INC}", f"-I{odir}", f"-I{sdir}", *src, "-o", out], verbose)
    return out


def build_all(force=False, verbose=False, gpu=True):
    outs = [build_prepro(force, verbose), build_oracle(force, verbose)]
    if gpu:
        outs.append(build_gpu(force, verbose))
    return outs


if __name__ == "__main__":
    for p in build_all(force="--force" in sys.argv, verbose=True):
        print("built", p)
