"""Builds the in-tree shared library libcfd_b200.so for sm_100a with nvcc.

The device code is compiled with --fmad=false so that every double operation is the separately
rounded IEEE operation the source states (the parity contract with the reference CPU code); the
host code (mesh geometry) is compiled without FMA contraction for the same reason.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libcfd_b200.so")
SOURCES = ["kernels.cu", "context.cu", "mesh.cpp", "json_config.cpp", "noalloc.cu", "mpnn.cu", "mpnn_tc.cu", "solution_io.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.sep not in c or os.path.exists(c)):
            return c
    return "nvcc"


def needs_build():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(ROOT, "include", "cfd_b200.h")]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False):
    if not force and not needs_build():
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    common = ["-std=c++17", "-O3", "-lineinfo", "--fmad=false", "-Xcompiler", "-fPIC,-ffp-contract=off",
              "-I" + os.path.join(ROOT, "include")] + ARCH
    objs = []
    procs = []
    for src in SOURCES:
        obj = os.path.join(objdir, os.path.splitext(src)[0] + ".o")
        cmd = [nvcc()] + common + ["-x", "cu" if src.endswith(".cu") else "c++", "-c", os.path.join(CSRC, src), "-o", obj]
        if os.environ.get("CFD_PTXAS_VERBOSE") and src.endswith(".cu"):
            cmd += ["-Xptxas", "-v"]
        procs.append((src, cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
        objs.append(obj)
    for src, cmd, p in procs:
        out, _ = p.communicate()
        if verbose or p.returncode != 0 or os.environ.get("CFD_PTXAS_VERBOSE"):
            sys.stderr.write(out)
        if p.returncode != 0:
            raise RuntimeError("nvcc failed on %s: %s" % (src, " ".join(cmd)))
    tmp = LIB + ".tmp"
    link = ["-Xlinker", "--version-script=" + os.path.join(CSRC, "exports.map"), "-Xlinker", "--exclude-libs,ALL"]
    subprocess.check_call([nvcc()] + ARCH + ["-shared", "-o", tmp] + objs + link + ["-lcudart"])
    os.replace(tmp, LIB)
    build_pybind()
    return LIB


def pybind_path():
    import sysconfig
    return os.path.join(HERE, "CFD_Solver" + sysconfig.get_config_var("EXT_SUFFIX"))


def build_pybind():
    """The Python module CFD_Solver (pybind/cfd_solver_module.cpp: the reference wrapper's
    interface over the C ABI), host code only, linked against libcfd_b200.so beside it."""
    import sysconfig
    try:
        import pybind11
    except ImportError:  # the module is optional; the ctypes binding covers the same calls
        return None
    out = pybind_path()
    cmd = ["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-I" + pybind11.get_include(),
           "-I" + sysconfig.get_paths()["include"], "-I" + os.path.join(ROOT, "include"),
           os.path.join(HERE, "pybind", "cfd_solver_module.cpp"), "-o", out + ".tmp", "-L" + HERE, "-lcfd_b200",
           "-Wl,-rpath,$ORIGIN"]
    subprocess.check_call(cmd)
    os.replace(out + ".tmp", out)
    return out


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
