"""Build recipe for the oracle (test infrastructure only).

* oracle/liboracle.so      -- the CPU restatement in elas_oracle.cpp, plus
  the seeded scene generator (cuda-stereo-matching_b200/csrc/synth.cpp,
  compiled from the same source as the product's copy) so that the CPU
  baseline and the reference arm of the benchmark load no product library
* oracle/_ref/libreftriangle.so -- the reference's own Triangle
  (src/triangle.cpp) compiled from the reference tree, with the C shim
  tri_ref_shim.cpp.
* oracle/_ref/libelasref.so -- the reference's own GPU pipeline
  (src/Elas.cu, src/Kernels/*.cu, src/triangle.cpp, unmodified, with the
  CPU Triangle path its default build takes) compiled for sm_100a with the C
  shim ref_elas_shim.cu.
The _ref libraries are built only where the reference tree is present; the
prebuilt files travel with the repository snapshot.  The reference's src/
directory is taken from the ref_src argument, else the ELAS_REFERENCE_SRC
environment variable, else the reference checkout this recipe was written
against (command line: python build_oracle.py [--force] [--ref-src DIR]).
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SYNTH = os.path.join(os.path.dirname(HERE), "cuda-stereo-matching_b200", "csrc", "synth.cpp")
DEFAULT_REF_SRC = "/root/reference/src"


def ref_src_dir(ref_src=None):
    return ref_src or os.environ.get("ELAS_REFERENCE_SRC") or DEFAULT_REF_SRC


def _run(cmd):
    subprocess.run(cmd, check=True)


def build_oracle(force=False):
    out = os.path.join(HERE, "liboracle.so")
    src = os.path.join(HERE, "elas_oracle.cpp")
    if force or not os.path.exists(out) or os.path.getmtime(out) < max(os.path.getmtime(src),
                                                                        os.path.getmtime(SYNTH)):
        _run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off",
              src, SYNTH, "-o", out, "-ldl"])
    return out


def build_ref(force=False, ref_src=None):
    REF_SRC = ref_src_dir(ref_src)
    out_dir = os.path.join(HERE, "_ref")
    out = os.path.join(out_dir, "libreftriangle.so")
    tri = os.path.join(REF_SRC, "triangle.cpp")
    if not os.path.exists(tri):
        return out if os.path.exists(out) else None
    os.makedirs(out_dir, exist_ok=True)
    shim = os.path.join(HERE, "tri_ref_shim.cpp")
    if force or not os.path.exists(out) or os.path.getmtime(out) < os.path.getmtime(shim):
        _run(["g++", "-O2", "-fPIC", "-shared", "-w", "-DREAL_TYPE_FP32", "-I" + REF_SRC,
              tri, shim, "-o", out])
    return out


def build_ref_elas(force=False, ref_src=None):
    REF_SRC = ref_src_dir(ref_src)
    out_dir = os.path.join(HERE, "_ref")
    out = os.path.join(out_dir, "libelasref.so")
    elas = os.path.join(REF_SRC, "Elas.cu")
    if not os.path.exists(elas):
        return out if os.path.exists(out) else None
    os.makedirs(out_dir, exist_ok=True)
    shim = os.path.join(HERE, "ref_elas_shim.cu")
    if force or not os.path.exists(out) or os.path.getmtime(out) < os.path.getmtime(shim):
        kernels = [os.path.join(REF_SRC, "Kernels", k) for k in
                   ("KerComputeDisparity.cu", "KerDescriptor.cu", "KerGrid.cu", "KerLeftRightConsistencyCheck.cu",
                    "KerSupportMatches.cu")]
        _run([os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc"), "-gencode", "arch=compute_100a,code=sm_100a",
              "-O2", "-std=c++14", "-Xcompiler", "-fPIC", "-shared", "-w", "-DREAL_TYPE_FP32", "-I" + REF_SRC,
              elas] + kernels + [os.path.join(REF_SRC, "triangle.cpp"), shim, "-o", out])
    return out


if __name__ == "__main__":
    force = "--force" in sys.argv
    src = sys.argv[sys.argv.index("--ref-src") + 1] if "--ref-src" in sys.argv else None
    print(build_oracle(force))
    print(build_ref(force, src))
    print(build_ref_elas(force, src))
