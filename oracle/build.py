"""Build recipe of the oracle libraries (test infrastructure only).

`build_oracle()` compiles the C++ restatement into oracle/liborc.so.
`build_reference()` compiles the reference's own device sources, in place,
into oracle/_ref/ with the shim and harnesses of oracle/ref/. Both run with
g++/nvcc only.
"""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
ORC_SO = os.path.join(HERE, "liborc.so")
REF_DIR = os.path.join(HERE, "_ref")
REF_SRC = os.environ.get("MRPNN_REFERENCE", "/root/reference")


def _newer(target, deps):
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps if os.path.exists(d))


def build_oracle(force=False):
    srcs = [os.path.join(HERE, "mr_oracle.cpp")]
    deps = srcs + [os.path.join(HERE, "mr_oracle_math.hpp"),
                   os.path.join(ROOT, "include", "mrpnn_b200.h"),
                   os.path.join(ROOT, "include", "mrpnn_weights.h")]
    if not force and _newer(ORC_SO, deps):
        return ORC_SO
    cmd = ["g++", "-std=c++17", "-O3", "-march=x86-64-v3", "-fopenmp", "-ffp-contract=off",
           "-fPIC", "-shared", "-o", ORC_SO] + srcs
    subprocess.check_call(cmd)
    return ORC_SO


def build_reference(force=False):
    """Compile the reference's device code (core/vector.cu, renderResources.cu,
    radiancePredict.cu via ref_net_tu.cu, render.cuh via the harness) for sm_100a into
    oracle/_ref/libref_mrpnn.so. Returns the path, or None when the reference
    sources are not present (e.g. on a GPU box)."""
    core = os.path.join(REF_SRC, "core")
    if not os.path.isdir(core):
        return None
    build_reference_volume(force)
    os.makedirs(REF_DIR, exist_ok=True)
    out = os.path.join(REF_DIR, "libref_mrpnn.so")
    ref_dir = os.path.join(HERE, "ref")
    shim = os.path.join(ref_dir, "cuda12_texref_shim.cuh")
    harness = os.path.join(ref_dir, "ref_harness.cu")
    net_tu = os.path.join(ref_dir, "ref_net_tu.cu")
    deps = [shim, harness, net_tu, os.path.join(ref_dir, "ref_inject.cu"),
            os.path.join(ROOT, "include", "mrpnn_weights.h")] + [os.path.join(core, f) for f in
                              ("vector.cu", "renderResources.cu", "radiancePredict.cu",
                               "render.cuh", "NNWeight.cuh")]
    if not force and _newer(out, deps):
        return out
    # The reference's stock CUDA flags (CMakeLists.txt: -use_fast_math
    # -maxrregcount=168), retargeted to sm_100a, relocatable device code.
    flags = ["-std=c++17", "-rdc=true", "-gencode", "arch=compute_100a,code=sm_100a",
             "-use_fast_math", "-maxrregcount=168", "-DLINUX", "-Xcompiler", "-fPIC",
             "-w", "-include", shim, "-I", core]
    objs = []
    for src in (os.path.join(core, "vector.cu"), os.path.join(core, "renderResources.cu"), net_tu, harness):
        o = os.path.join(REF_DIR, os.path.basename(src).replace(".cu", ".o"))
        subprocess.check_call(["nvcc"] + flags + ["-c", src, "-o", o])
        objs.append(o)
    subprocess.check_call(["nvcc", "-shared", "-gencode", "arch=compute_100a,code=sm_100a",
                           "-Xcompiler", "-fPIC", "-o", out] + objs)
    # Descriptor-injection build of the network (reference option
    # DISABLE_FAST_MATH, i.e. without -use_fast_math).
    inj = os.path.join(ref_dir, "ref_inject.cu")
    iflags = [f for f in flags if f != "-use_fast_math"] + ["-DMR_REF_INJECT"]
    iobjs = []
    for src in (os.path.join(core, "vector.cu"), net_tu, inj):
        o = os.path.join(REF_DIR, "inj_" + os.path.basename(src).replace(".cu", ".o"))
        subprocess.check_call(["nvcc"] + iflags + ["-c", src, "-o", o])
        iobjs.append(o)
    subprocess.check_call(["nvcc", "-shared", "-gencode", "arch=compute_100a,code=sm_100a",
                           "-Xcompiler", "-fPIC", "-o", os.path.join(REF_DIR, "libref_net_inj.so")]
                          + iobjs)
    return out


def build_reference_volume(force=False):
    """Compile the reference's VolumeRender (core/volume.cu with camera.cu,
    omp.cpp, vector.cu, renderResources.cu and radiancePredict.cu) with the
    harness oracle/ref/ref_volume.cu into oracle/_ref/libref_volume.so."""
    core = os.path.join(REF_SRC, "core")
    if not os.path.isdir(core):
        return None
    os.makedirs(REF_DIR, exist_ok=True)
    out = os.path.join(REF_DIR, "libref_volume.so")
    ref_dir = os.path.join(HERE, "ref")
    shim = os.path.join(ref_dir, "cuda12_texref_shim.cuh")
    harness = os.path.join(ref_dir, "ref_volume.cu")
    datagen = os.path.join(ref_dir, "ref_datagen.cu")
    net_tu = os.path.join(ref_dir, "ref_net_tu.cu")
    srcs = [os.path.join(core, f) for f in ("vector.cu", "renderResources.cu", "volume.cu", "camera.cu")]
    deps = [shim, harness, datagen, net_tu, os.path.join(REF_SRC, "dataGen.cu")] + srcs + [
        os.path.join(core, f) for f in ("omp.cpp", "render.cuh", "volume.hpp", "camera.hpp", "NNWeight.cuh")]
    if not force and _newer(out, deps):
        return out
    flags = ["-std=c++17", "-rdc=true", "-gencode", "arch=compute_100a,code=sm_100a",
             "-use_fast_math", "-maxrregcount=168", "-DLINUX", "-Xcompiler", "-fPIC",
             "-w", "-include", shim, "-I", core]
    objs = []
    for src in srcs + [net_tu, harness]:
        o = os.path.join(REF_DIR, "vol_" + os.path.basename(src).replace(".cu", ".o"))
        subprocess.check_call(["nvcc"] + flags + ["-c", src, "-o", o])
        objs.append(o)
    # dataGen.cu (its sampling functions): the GUI header it includes is
    # replaced by a stub, its main renamed inside ref_datagen.cu
    o = os.path.join(REF_DIR, "vol_ref_datagen.o")
    subprocess.check_call(["nvcc"] + flags[:-2] + ["-I", os.path.join(ref_dir, "stub"), "-I", core, "-I", REF_SRC,
                                                   "-c", datagen, "-o", o])
    objs.append(o)
    o = os.path.join(REF_DIR, "vol_omp.o")
    subprocess.check_call(["nvcc", "-std=c++17", "-w", "-Xcompiler", "-fPIC", "-gencode",
                           "arch=compute_100a,code=sm_100a", "-I", core, "-x", "cu", "-c",
                           os.path.join(core, "omp.cpp"), "-o", o])
    objs.append(o)
    subprocess.check_call(["nvcc", "-shared", "-gencode", "arch=compute_100a,code=sm_100a",
                           "-Xcompiler", "-fPIC", "-o", out] + objs)
    return out


if __name__ == "__main__":
    print(build_oracle(force=True))
    print(build_reference(force=True))
