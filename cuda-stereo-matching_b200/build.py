"""Build the ELAS B200 library in-tree: libelas_b200.so next to this file.

Every CUDA source is compiled for sm_100a only
(-gencode arch=compute_100a,code=sm_100a) with line info; the host sources
(synthetic scenes) are compiled by the same nvcc invocation's host compiler.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libelas_b200.so")
CLI = os.path.join(HERE, "elas_b200_cli")
CLI_SOURCES = [os.path.join(HERE, "cli", "elas_cli.cpp"), os.path.join(HERE, "cli", "pnm_io.h")]
OBJ_DIR = os.path.join(HERE, "_build")

CU_SOURCES = ["k_descriptor.cu", "k_support.cu", "k_delaunay.cu", "k_dense.cu", "k_post.cu", "k_proposal.cu",
              "k_proposal_tc.cu", "elas_api.cu"]
CPP_SOURCES = ["synth.cpp", "elas_group.cpp"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fopenmp"]


def _stale(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False, ptxas_info=False):
    os.makedirs(OBJ_DIR, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(HERE, "..", "include", "elas_b200.h"))
    objs = []
    for src in CU_SOURCES + CPP_SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(OBJ_DIR, src + ".o")
        objs.append(obj)
        if force or _stale(obj, [path] + headers):
            cmd = [NVCC] + ARCH + COMMON + ["-c", path, "-o", obj]
            if src.endswith(".cpp"):
                cmd = [NVCC, "-Wno-deprecated-gpu-targets"] + COMMON + ["-Xcompiler", "-pthread", "-x", "c++", "-c",
                                                                        path, "-o", obj]
            if ptxas_info and src.endswith(".cu"):
                cmd.insert(1, "-Xptxas=-v")
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
    if force or _stale(OUT, objs):
        # link beside the library and rename it into place, so that a reader
        # never sees a partly written file
        tmp = OUT + ".tmp"
        cmd = [NVCC] + ARCH + ["-shared", "-o", tmp] + objs + ["-lgomp", "-lpthread"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        os.replace(tmp, OUT)
    # the command-line front end (host code linked against the library)
    if force or _stale(CLI, CLI_SOURCES + [OUT, os.path.join(HERE, "..", "include", "elas_b200.h")]):
        cmd = ["g++", "-O2", "-std=c++17", "-I", os.path.join(HERE, "..", "include"), CLI_SOURCES[0], "-o", CLI,
               "-L", HERE, "-lelas_b200", "-Wl,-rpath,$ORIGIN"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv, ptxas_info="--ptxas" in sys.argv))
