"""Builds libimpz_b200.so (sm_100a) in place, and the CPU oracle used by the tests.

    python impact-z_b200/build.py            # library + oracle
    python impact-z_b200/build.py --lib      # library only

nvcc cross-compiles for sm_100a without a GPU.  The plain-FP64 particle
kernels and the Poisson solve are compiled with --fmad=false so their FP64
arithmetic rounds like the reference's x86-64 build; the FP32-convolution
particle kernels may contract.  Host numerics are built with
-ffp-contract=off for the same reason.
"""
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libimpz_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_COMMON = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                      "-Xcompiler", "-ffp-contract=off", "-I", CSRC]

# (source, extra flags)
UNITS = [
    ("impz_particle_exact.cu", ["--fmad=false"]),
    ("impz_particle_fast.cu", []),
    ("impz_poisson.cu", ["--fmad=false"]),
    ("impz_capi.cu", []),
    ("impz_serve.cu", []),
    ("impz_static.cu", ["--fmad=false"]),
]
HOST_UNITS = ["impz_host.cpp"]


def nvcc():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def host_cxx():
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed: %s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr))
    return r.stdout + r.stderr


def _newer(target, deps):
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps)


def _deps(src):
    hdrs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hdrs.append(os.path.join(ROOT, "include", "impz_b200.h"))
    return [src] + hdrs + [os.path.abspath(__file__)]


def build_lib(verbose=False, defines=(), lib=None, obj=None):
    """Builds the library; `defines` (e.g. ["-DIMPZ_ADV_U=2"]) and an
    alternative output path allow side-by-side launch-shape variants."""
    global OBJ
    lib = lib or LIB
    obj_dir = obj or OBJ
    os.makedirs(obj_dir, exist_ok=True)
    saved, OBJ = OBJ, obj_dir
    try:
        return _build_lib(verbose, list(defines), lib)
    finally:
        OBJ = saved


def _build_lib(verbose, defines, lib_path):
    nv = nvcc()
    jobs = []
    objs = []
    for src, extra in UNITS:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src + ".o")
        objs.append(o)
        if not _newer(o, _deps(s)):
            jobs.append([nv] + NVCC_COMMON + extra + defines + ["-c", s, "-o", o])
    for src in HOST_UNITS:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src + ".o")
        objs.append(o)
        if not _newer(o, _deps(s)):
            jobs.append([host_cxx(), "-O2", "-std=c++17", "-fPIC", "-ffp-contract=off",
                         "-I", CSRC, "-c", s, "-o", o])
    with cf.ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 4))) as ex:
        for out in ex.map(_run, jobs):
            if verbose and out.strip():
                print(out)
    if jobs or not os.path.exists(lib_path):
        _run([nv] + ARCH + ["-shared", "-o", lib_path] + objs + ["-lcudart_static", "-lrt",
                                                                  "-ldl", "-lpthread"])
    return lib_path


def build_oracle():
    odir = os.path.join(ROOT, "oracle")
    _run(["make", "-s", "-C", odir])
    return os.path.join(odir, "liboracle_impz.so")


if __name__ == "__main__":
    lib = build_lib(verbose="-v" in sys.argv)
    print(lib)
    if "--lib" not in sys.argv:
        print(build_oracle())
