"""Build the native parts of the engine in-tree.

    python parallelac-xmp_b200/build.py          # incremental
    python parallelac-xmp_b200/build.py --clean  # from scratch

Outputs (git-ignored, shipped with the tree):
    parallelac-xmp_b200/lib/libpac.so          the C ABI of include/pac.h
    parallelac-xmp_b200/lib/libpac_synth.so    seeded workload generators
    parallelac-xmp_b200/bin/parallelac         CLI, plain-xmp formulas
    parallelac-xmp_b200/bin/parallelac-largeData  CLI, upstream formulas

The device code is compiled for sm_100a only.  pipeline.cu is compiled twice,
once per arithmetic flavour (see csrc/refarith.cuh).
"""
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(PKG, "csrc")
INC = os.path.join(os.path.dirname(PKG), "include")
OBJ = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "lib")
BIN = os.path.join(PKG, "bin")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
HOSTCC = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
HOSTC = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                  "-ccbin", HOSTCC, "-I", INC, "--expt-relaxed-constexpr"]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("command failed: %s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr))
    return r.stdout + r.stderr


def _stale(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def _headers():
    return [os.path.join(SRC, f) for f in os.listdir(SRC)
            if f.endswith((".h", ".cuh"))] + [os.path.join(INC, "pac.h")]


def build(verbose=False, ptxas_info=False):
    for d in (OBJ, LIB, BIN):
        os.makedirs(d, exist_ok=True)
    hdrs = _headers()
    extra = ["-Xptxas", "-v"] if ptxas_info else []
    jobs = [
        (os.path.join(OBJ, "pipeline_strict.o"),
         [NVCC] + NVFLAGS + extra + ["-fmad=false", "-DPAC_NS=pac_strict", "-DPAC_WITH_EXACT=1", "-c",
                                     os.path.join(SRC, "pipeline.cu")],
         [os.path.join(SRC, "pipeline.cu")] + hdrs),
        (os.path.join(OBJ, "pipeline_fma.o"),
         [NVCC] + NVFLAGS + extra + ["-fmad=true", "-DPAC_NS=pac_fma", "-c",
                                     os.path.join(SRC, "pipeline.cu")],
         [os.path.join(SRC, "pipeline.cu")] + hdrs),
        (os.path.join(OBJ, "union_measure.o"),
         [NVCC] + NVFLAGS + extra + ["-c", os.path.join(SRC, "union_measure.cu")],
         [os.path.join(SRC, "union_measure.cu")] + hdrs),
        (os.path.join(OBJ, "engine.o"),
         [NVCC] + NVFLAGS + extra + ["-c", os.path.join(SRC, "engine.cu")],
         [os.path.join(SRC, "engine.cu")] + hdrs),
        (os.path.join(OBJ, "textio.o"),
         [HOSTCC, "-O2", "-std=c++17", "-fPIC", "-pthread", "-I", INC, "-c",
          os.path.join(SRC, "textio.cpp")],
         [os.path.join(SRC, "textio.cpp"), os.path.join(INC, "pac.h")]),
    ]
    todo = [(o, c + ["-o", o]) for o, c, deps in jobs if _stale(o, deps)]
    logs = []
    with ThreadPoolExecutor(max_workers=4) as ex:
        for out in ex.map(lambda oc: _run(oc[1]), todo):
            logs.append(out)
    objs = [o for o, _, _ in jobs]
    lib = os.path.join(LIB, "libpac.so")
    if _stale(lib, objs):
        _run([NVCC] + ARCH + ["-shared", "-cudart", "static", "-ccbin", HOSTCC, "-o", lib] + objs +
             ["-lpthread"])
    synth = os.path.join(LIB, "libpac_synth.so")
    if _stale(synth, [os.path.join(SRC, "synth.c")]):
        _run([HOSTC, "-O2", "-std=c99", "-fPIC", "-shared", "-o", synth,
              os.path.join(SRC, "synth.c"), "-lm"])
    for name, defs in (("parallelac", []), ("parallelac-largeData", ["-DPAC_CLI_LARGEDATA"])):
        exe = os.path.join(BIN, name)
        if _stale(exe, [os.path.join(SRC, "cli.cpp"), lib]):
            _run([HOSTCC, "-O2", "-std=c++17"] + defs + ["-I", INC, "-o", exe,
                  os.path.join(SRC, "cli.cpp"), "-L", LIB, "-lpac",
                  "-Wl,-rpath,$ORIGIN/../lib"])
    if verbose:
        for l in logs:
            sys.stdout.write(l)
    return "\n".join(logs)


if __name__ == "__main__":
    if "--clean" in sys.argv:
        for d in (OBJ, LIB, BIN):
            shutil.rmtree(d, ignore_errors=True)
    print(build(verbose="-v" in sys.argv, ptxas_info="--ptxas" in sys.argv) or "up to date")
