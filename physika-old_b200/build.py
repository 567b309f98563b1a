"""Builds libpkhot.so (sm_100a) in-tree.  Incremental: skips when up to date."""
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CU_SOURCES = ["pk_sort.cu", "pk_nbr.cu", "pk_pbd.cu", "pk_pd.cu", "pk_pd_adj.cu", "pk_fixed.cu", "pk_plastic.cu", "pk_pbd_adj.cu", "pk_api.cu",
              "pk_noalloc.cu"]


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build_pkhot(force=False, verbose=True):
    out = os.path.join(HERE, "lib", "libpkhot.so")
    srcs = [os.path.join(HERE, "csrc", s) for s in CU_SOURCES]
    deps = srcs + glob.glob(os.path.join(HERE, "csrc", "*.cuh")) + [
        os.path.join(ROOT, "include", "pk_hot.h")]
    if not force and not _newer(out, deps):
        return out
    os.makedirs(os.path.dirname(out), exist_ok=True)
    cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17",
           "-Xcompiler", "-fPIC,-fvisibility=hidden,-ffp-contract=off",
           "-shared", "-o", out + ".tmp", *srcs]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(out + ".tmp", out)
    return out


def build_framework(force=False, verbose=True):
    """The C++ Framework mirror (framework/*.cpp: the reference-named modules
    and the headless scene driver) into lib/libpkframework.so, linked against
    libpkhot.so (found next to it at run time)."""
    out = os.path.join(HERE, "lib", "libpkframework.so")
    fw = os.path.join(HERE, "framework")
    srcs = [os.path.join(fw, s) for s in ("ParticleModules.cpp", "ParticleIO.cpp", "scene_driver.cpp")]
    deps = srcs + glob.glob(os.path.join(fw, "*.h")) + [os.path.join(ROOT, "include", "pk_hot.h")]
    if not force and not _newer(out, deps):
        return out
    cuda = os.path.dirname(os.path.dirname(NVCC))
    cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-fvisibility=hidden", "-Wall",
           "-I", os.path.join(ROOT, "include"), "-I", os.path.join(cuda, "include"), *srcs,
           "-L", os.path.join(HERE, "lib"), "-lpkhot", "-L", os.path.join(cuda, "lib64"), "-lcudart",
           "-Wl,-rpath,$ORIGIN", "-Wl,-rpath," + os.path.join(cuda, "lib64"), "-o", out + ".tmp"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(out + ".tmp", out)
    return out


def pkbind_path():
    import sysconfig
    return os.path.join(HERE, "lib", "_pkbind" + sysconfig.get_config_var("EXT_SUFFIX"))


def build_pkbind(force=False, verbose=True):
    """The pybind11 layer of the differentiable rollouts (csrc/pk_pybind.cpp)
    into lib/_pkbind*.so, linked against libpkhot.so (found next to it)."""
    import sysconfig
    import pybind11
    out = pkbind_path()
    src = os.path.join(HERE, "csrc", "pk_pybind.cpp")
    deps = [src, os.path.join(ROOT, "include", "pk_hot.h")]
    if not force and not _newer(out, deps):
        return out
    cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-fvisibility=hidden", "-Wall",
           "-I", pybind11.get_include(), "-I", sysconfig.get_paths()["include"], src,
           "-L", os.path.join(HERE, "lib"), "-lpkhot", "-Wl,-rpath,$ORIGIN", "-o", out + ".tmp"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(out + ".tmp", out)
    return out


# The reference checkout: PK_REFERENCE_SRC, else a directory named `reference`
# beside this repository.  Only the golden-fixture drivers under oracle/_ref
# need it; a machine without it uses the prebuilt drivers.
REFERENCE = os.environ.get("PK_REFERENCE_SRC") or os.path.join(os.path.dirname(ROOT), "reference")


def build_oracle(verbose=True, with_ref=False):
    """The CPU restatement; with_ref also builds the golden-fixture drivers from
    the reference sources when they are present: oracle/_ref/ref_math_probe
    (its vector math and kernel weights) and oracle/_ref/pkref_driver (its own
    NeighborQuery, SummationDensity, DensityPBD, ParticleIntegrator and
    ElasticityModule kernels)."""
    out = None if verbose else subprocess.DEVNULL
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True, stdout=out)
    if with_ref and os.path.isdir(os.path.join(REFERENCE, "Source")):
        subprocess.run(["make", "-s", "-j8", "-C", os.path.join(ROOT, "oracle"), "ref", "refk", "REF=" + REFERENCE],
                       check=True, stdout=out)


if __name__ == "__main__":
    build_pkhot(force="--force" in sys.argv)
    build_framework(force="--force" in sys.argv)
    build_pkbind(force="--force" in sys.argv)
    build_oracle(with_ref=True)
