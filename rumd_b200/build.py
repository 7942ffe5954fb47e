"""Builds the native parts of rumd_b200 in-tree for sm_100a.

  librumd_b200.so   CUDA kernels + engine + C ABI (include/rumd_b200.h)
  _rumd*.so         pybind11 module with the RUMD class surface (Sample,
                    Pot_LJ_12_6, IntegratorNVT, ...), linked to librumd_b200.so

Run ``python -m rumd_b200.build`` or call ``build()``.
"""
import os
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "librumd_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def _newer(target, sources):
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(s) <= t for s in sources)


def _sources(exts):
    out = []
    for d in (CSRC, os.path.join(CSRC, "rumd"), os.path.join(ROOT, "include")):
        if os.path.isdir(d):
            out += [os.path.join(d, f) for f in os.listdir(d) if f.endswith(exts)]
    return out


def build_lib(force=False):
    cu = [os.path.join(CSRC, "engine.cu"), os.path.join(CSRC, "probe.cu"), os.path.join(CSRC, "noalloc.cu"),
          os.path.join(CSRC, "f64.cu")]
    deps = _sources((".cu", ".cuh", ".h"))
    if not force and _newer(LIB, deps):
        return LIB
    _run([NVCC, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-shared", "-Xcompiler", "-fPIC",
          "-Xcompiler", "-fvisibility=hidden", "-Xcompiler", "-Wall", *cu, "-o", LIB])
    return LIB


def module_path():
    suffix = sysconfig.get_config_var("EXT_SUFFIX") or ".so"
    return os.path.join(HERE, "_rumd" + suffix)


def build_module(force=False):
    src = os.path.join(CSRC, "pymodule.cpp")
    if not os.path.exists(src):
        return None
    out = module_path()
    deps = _sources((".cpp", ".h")) + [LIB]
    if not force and _newer(out, deps):
        return out
    import pybind11
    cpp = [src, os.path.join(CSRC, "rumd", "rumd_classes.cpp")]
    inc = ["-I" + pybind11.get_include(), "-I" + sysconfig.get_paths()["include"],
           "-I" + os.path.join(ROOT, "include"), "-I" + CSRC, "-I/usr/local/cuda/include"]
    _run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-fvisibility=hidden", "-Wall",
          *inc, *cpp, "-L" + HERE, "-lrumd_b200", "-Wl,-rpath,$ORIGIN", "-lz", "-o", out])
    return out


def build(force=False):
    build_lib(force)
    build_module(force)


if __name__ == "__main__":
    build(force="--force" in sys.argv)
