"""Builds libx2.so in-tree for sm_100a (nvcc), next to the Python layer in x2/.

The CUDA sources are compiled without floating-point contraction (-fmad=false): the path arithmetic is
written to round exactly as the reference's CPU lane (-ffp-contract=off) does, and the parity tests rely on it.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "x2", "libx2.so")
# The diagnostic build (parity investigation only, never the product): render.cu compiled with -DX2_DIAG (mathfn.cuh:
# transcendental functions in double on request, and a record of every call), linked with the product's other objects.
DIAG_OUT = os.path.join(HERE, "x2", "libx2diag.so")
# The contracted build (a measurement, never the product): the render and wavefront kernels compiled with -fmad=true,
# as the reference's production GPU lane is built, to report that speed beside the parity build's.
FMAD_OUT = os.path.join(HERE, "x2", "libx2fmad.so")
FMAD_CU = ["render.cu", "wavefront.cu"]
BUILD = os.path.join(HERE, "_build")
CU = ["api.cu", "render.cu", "wavefront.cu", "bvh_build.cu", "noalloc.cu", "adjoint.cu", "adaptive.cu", "scores.cu", "probe.cu"]
CPP = ["scene_gen.cpp", "grid.cpp"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-fmad=false", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-Xptxas", "-warn-spills"]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("build failed: " + " ".join(cmd))
    return r.stdout + r.stderr


def _stale(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def build(verbose=False, force=False):
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(HERE, "..", "include", "x2.h"))
    objs = []
    for f in CU:
        src = os.path.join(CSRC, f)
        obj = os.path.join(BUILD, f + ".o")
        if force or _stale(obj, [src] + headers):
            log = _run([NVCC] + ARCH + FLAGS + ["-rdc=false", "-c", src, "-o", obj] + (["-Xptxas", "-v"] if verbose else []))
            if verbose:
                sys.stdout.write(log)
        objs.append(obj)
    for f in CPP:
        src = os.path.join(CSRC, f)
        obj = os.path.join(BUILD, f + ".o")
        if force or _stale(obj, [src] + headers):
            _run(["g++", "-std=c++17", "-O2", "-fPIC", "-c", src, "-o", obj])
        objs.append(obj)
    if force or _stale(OUT, objs):
        _run([NVCC] + ARCH + ["-shared", "-Xcompiler", "-fPIC", "-o", OUT] + objs + ["-lcudart_static"])
    diag = os.path.join(BUILD, "render_diag.cu.o")
    src = os.path.join(CSRC, "render.cu")
    if force or _stale(diag, [src] + headers + [os.path.join(HERE, "..", "include", "x2_diag.h")]):
        _run([NVCC] + ARCH + FLAGS + ["-DX2_DIAG", "-rdc=false", "-c", src, "-o", diag])
    diag_objs = [diag if o.endswith(os.sep + "render.cu.o") else o for o in objs]
    if force or _stale(DIAG_OUT, diag_objs):
        _run([NVCC] + ARCH + ["-shared", "-Xcompiler", "-fPIC", "-o", DIAG_OUT] + diag_objs + ["-lcudart_static"])
    fmad_objs = []
    for o in objs:
        name = os.path.basename(o)[:-2]  # "<file>.cu"
        if name in FMAD_CU:
            fo = os.path.join(BUILD, name + ".fmad.o")
            src = os.path.join(CSRC, name)
            if force or _stale(fo, [src] + headers):
                _run([NVCC] + ARCH + [f if f != "-fmad=false" else "-fmad=true" for f in FLAGS] + ["-rdc=false", "-c", src, "-o", fo])
            fmad_objs.append(fo)
        else:
            fmad_objs.append(o)
    if force or _stale(FMAD_OUT, fmad_objs):
        _run([NVCC] + ARCH + ["-shared", "-Xcompiler", "-fPIC", "-o", FMAD_OUT] + fmad_objs + ["-lcudart_static"])
    return OUT


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
