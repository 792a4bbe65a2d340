"""Build libnecpp_b200.so in-tree: host C++ (g++) + sm_100a CUDA (nvcc).

The host library is compiled with -ffp-contract=off so the geometry,
connection and basis-coefficient arithmetic rounds exactly as the reference's
x86-64 build does.  CUDA code is compiled for sm_100a only.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libnecpp_b200.so")

HOST_SRCS = ["geometry.cpp", "context.cpp", "c_api.cpp", "deck.cpp"]
CLI_SRC = "nec2b200_main.cpp"
CLI = os.path.join(HERE, "nec2b200")
CUDA_SRCS = ["engine.cu"]
CUDA_ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _cxx():
    # the system compiler links libstdc++ dynamically; a toolchain that links
    # a private static copy clashes with the libstdc++ numpy/torch load
    if os.path.exists("/usr/bin/g++"):
        return "/usr/bin/g++"
    return shutil.which("g++") or "g++"


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    inc = os.path.join(os.path.dirname(HERE), "include")
    hs += [os.path.join(inc, f) for f in os.listdir(inc) if f.endswith(".h")]
    return hs


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError("build step failed: " + os.path.basename(cmd[-1]))
    return r


def build(verbose=False, force=False):
    os.makedirs(OBJ, exist_ok=True)
    heads = _headers()
    objs = []
    for src in HOST_SRCS:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src + ".o")
        if force or _newer(o, [s] + heads):
            _run([_cxx(), "-std=c++17", "-O2", "-fPIC", "-ffp-contract=off", "-fno-fast-math",
                  "-Wall", "-Wextra", "-Wno-unused-parameter", "-I", os.path.join(HERE, ".."),
                  "-c", s, "-o", o])
        objs.append(o)
    nvcc = _nvcc()
    for src in CUDA_SRCS:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src + ".o")
        if force or _newer(o, [s] + heads):
            _run([nvcc] + CUDA_ARCH + ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC",
                                       "-Xptxas", "-v" if verbose else "-O3", "-c", s, "-o", o])
        objs.append(o)
    if force or _newer(LIB, objs):
        _run([nvcc] + CUDA_ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs)
    # the deck-file command line (nec2++'s -i / -o), linked to the library
    cli_src = os.path.join(CSRC, CLI_SRC)
    if force or _newer(CLI, [cli_src, LIB]):
        _run([_cxx(), "-std=c++17", "-O2", "-I", os.path.join(HERE, ".."), cli_src, "-o", CLI,
              "-L", HERE, "-lnecpp_b200", "-Wl,-rpath,$ORIGIN"])
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
