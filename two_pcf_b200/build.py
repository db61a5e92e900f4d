"""Builds the engine in-tree: two_pcf_b200/lib/libtpcf_b200.so (C ABI of
include/two_pcf_b200.h) for sm_100a only, plus the command-line driver.

Host C++ is compiled with -ffp-contract=off: the threshold tables and the
cosmology table must round every float/double operation once, like the
reference's x86-64 build.

TPCF_DEVICE_CHECKS=1 (or build(checked=True)) builds the checked library
instead: every count kernel tests its indices against their bounds (see
tpcf_device_checks in include/two_pcf_b200.h); objects in lib/obj-checked,
library lib/checked/libtpcf_b200.so, loaded when TPCF_CHECKED=1.

TPCF_SANITIZE=1 builds the host C++ with AddressSanitizer and
UndefinedBehaviorSanitizer instead (objects in lib/obj-sanitize; the library
is relinked whenever the mode changes).  Python is not instrumented, so run
with the runtime preloaded, e.g.
  LD_PRELOAD=$(gcc -print-file-name=libasan.so) ASAN_OPTIONS=detect_leaks=0 \
      python -m pytest tests -m "not gpu"
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB_DIR = os.path.join(PKG, "lib")
SANITIZE = os.environ.get("TPCF_SANITIZE", "") == "1"
BUILD_DIR = os.path.join(PKG, "lib", "obj-sanitize" if SANITIZE else "obj")
LIB_PATH = os.path.join(LIB_DIR, "libtpcf_b200.so")
SAN_FLAGS = ["-fsanitize=address,undefined", "-fno-omit-frame-pointer", "-g"]

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
CXX = os.environ.get("TPCF_CXX", "g++")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

CU_SOURCES = ["grid.cu", "pair_count.cu", "diag.cu"]
CPP_SOURCES = ["axis.cpp", "capi.cpp", "worklist.cpp", "ingest.cpp", "capi_host.cpp", "driver.cpp"]
CLI_SOURCE = "two_pcf_main.cpp"
CLI_PATH = os.path.join(LIB_DIR, "two_pcf")


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r.stdout + r.stderr


def _stale(obj, srcs):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(s) > t for s in srcs)


def build(verbose: bool = False, ptxas_info: bool = False, checked: bool | None = None) -> str:
    if checked is None:
        checked = os.environ.get("TPCF_DEVICE_CHECKS", "") == "1"
    build_dir = os.path.join(LIB_DIR, "obj-checked") if checked else BUILD_DIR
    lib_path = os.path.join(LIB_DIR, "checked", "libtpcf_b200.so") if checked else LIB_PATH
    defs = ["-DTPCF_DEVICE_CHECKS"] if checked else []
    os.makedirs(build_dir, exist_ok=True)
    os.makedirs(os.path.dirname(lib_path), exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(ROOT, "include", "two_pcf_b200.h"))
    jobs = []
    objs = []
    for f in CU_SOURCES:
        src = os.path.join(CSRC, f)
        obj = os.path.join(build_dir, f + ".o")
        objs.append(obj)
        if _stale(obj, [src] + headers):
            cmd = [NVCC, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC,-ffp-contract=off,-fopenmp",
                   *defs, "-I", CSRC, "-c", src, "-o", obj]
            if ptxas_info:
                cmd.insert(1, "-Xptxas=-v")
            jobs.append(cmd)
    for f in CPP_SOURCES:
        src = os.path.join(CSRC, f)
        obj = os.path.join(build_dir, f + ".o")
        objs.append(obj)
        if _stale(obj, [src] + headers):
            jobs.append([CXX, *(["-O1", *SAN_FLAGS] if SANITIZE else ["-O2"]), "-std=c++17", "-fPIC",
                         "-ffp-contract=off", "-fopenmp", *defs, "-I", CSRC,
                         "-I", os.path.join(CUDA_HOME, "include"), "-c", src, "-o", obj])
    with ThreadPoolExecutor(max_workers=max(1, os.cpu_count() or 1)) as ex:
        outs = list(ex.map(_run, jobs))
    if verbose:
        for o in outs:
            sys.stdout.write(o)
    mode = "sanitize" if SANITIZE else "release"
    stamp = os.path.join(os.path.dirname(lib_path), ".build_mode")
    last_mode = open(stamp).read().strip() if os.path.exists(stamp) else "release"
    if jobs or not os.path.exists(lib_path) or mode != last_mode:
        tmp = lib_path + ".tmp"
        if SANITIZE:
            _run([NVCC, *ARCH, "-shared", "-Xcompiler", "-fPIC,-fsanitize=address,-fsanitize=undefined", *objs,
                  "-o", tmp, "-lcudart_static", "-lgomp", "-lasan", "-lubsan"])
        else:
            _run([NVCC, *ARCH, "-shared", "-Xcompiler", "-fPIC", *objs, "-o", tmp, "-lcudart_static", "-lgomp"])
        shutil.move(tmp, lib_path)
        with open(stamp, "w") as f:
            f.write(mode + "\n")
    if checked:
        return lib_path
    cli_src = os.path.join(CSRC, CLI_SOURCE)
    if _stale(CLI_PATH, [cli_src, LIB_PATH] + headers):
        tmp = CLI_PATH + ".tmp"
        _run([CXX, "-O2", "-std=c++17", cli_src, "-o", tmp, "-L", LIB_DIR, "-ltpcf_b200", "-Wl,-rpath,$ORIGIN"])
        shutil.move(tmp, CLI_PATH)
    return LIB_PATH


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, ptxas_info="--ptxas" in sys.argv))
