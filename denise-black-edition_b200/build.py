"""Builds the in-tree native library and tools of the B200 P-SV propagator.

    python denise-black-edition_b200/build.py        # lib/libdenise_b200.so and bin/denise_b200

The CUDA sources are compiled for sm_100a only.  Host C set-up code is
compiled with -ffp-contract=off -fno-fast-math because it must reproduce
the reference's float/double rounding bit for bit.
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
HOST = os.path.join(HERE, "host")
LIB = os.path.join(HERE, "lib")
BIN = os.path.join(HERE, "bin")
BUILD = os.path.join(HERE, "_build")
INC = os.path.join(ROOT, "include")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
# extra nvcc flags, e.g. a kernel tuning macro for a measurement build (-DDN_PF2_ROWS=4)
EXTRA_NVCC = os.environ.get("DN_NVCC_FLAGS", "").split()
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
HOST_CFLAGS = ["-O2", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-Wall", "-Wno-unused-function"]

CU_SOURCES = ["dn_engine.cu", "dn_alloc.cu", "dn_residual.cu", "dn_fwi.cu", "dn_precond.cu", "dn_tdfilt.cu"] + [f"dn_launch_r{r}.cu" for r in range(1, 7)]
C_SOURCES = ["dn_setup.c", "dn_opt.c", "dn_precond_host.c"]
HOST_SOURCES = ["dn_io.c", "dn_driver.c"]
CLI_SOURCES = ["denise_b200_main.c"]


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=True):
    os.makedirs(LIB, exist_ok=True)
    os.makedirs(BIN, exist_ok=True)
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers += [os.path.join(INC, "denise_b200.h")]
    if os.path.isdir(HOST):
        headers += [os.path.join(HOST, f) for f in os.listdir(HOST) if f.endswith(".h")]
    objs, jobs = [], []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        if _newer(o, [s] + headers):
            jobs.append([NVCC] + ARCH + EXTRA_NVCC + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-ffp-contract=off",
                                         "-I", INC, "-I", CSRC, "-c", s, "-o", o])
        objs.append(o)
    # the CUDA translation units are independent: compile them concurrently
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        list(ex.map(_run, jobs))
    for d, srcs in ((CSRC, C_SOURCES), (HOST, HOST_SOURCES)):
        for src in srcs:
            s = os.path.join(d, src)
            if not os.path.exists(s):
                continue
            o = os.path.join(BUILD, src + ".o")
            if _newer(o, [s] + headers):
                _run(["gcc"] + HOST_CFLAGS + ["-I", INC, "-I", CSRC, "-I", HOST, "-c", s, "-o", o])
            objs.append(o)
    lib = os.path.join(LIB, "libdenise_b200.so")
    if _newer(lib, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", lib] + objs + ["-lcudart", "-lm"])
    for src in CLI_SOURCES:
        s = os.path.join(HOST, src)
        if not os.path.exists(s):
            continue
        exe = os.path.join(BIN, "denise_b200")
        if _newer(exe, [s, lib] + headers):
            _run(["gcc"] + HOST_CFLAGS + ["-I", INC, "-I", CSRC, "-I", HOST, s, "-o", exe,
                                          "-L", LIB, "-ldenise_b200", "-Wl,-rpath,$ORIGIN/../lib", "-lm"])
    # the per-kernel drop-ins with the reference's signatures: their own library, whose
    # undefined symbols (the reference's globals and err) resolve in the reference program
    shim_src = os.path.join(CSRC, "dn_fd_shims.cu")
    shim = os.path.join(LIB, "libdenise_b200_fd.so")
    if os.path.exists(shim_src) and _newer(shim, [shim_src] + headers):
        _run([NVCC] + ARCH + EXTRA_NVCC + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-ffp-contract=off",
                                           "-shared", "-I", INC, "-I", CSRC, shim_src, "-o", shim, "-lcudart"])
    return lib


if __name__ == "__main__":
    build()
    sys.exit(0)
