"""Build libgp (the C-ABI shared library over the sm_100a kernels) in-tree.

    python -m eshwar_dipan_b200.build [--verbose]

Outputs eshwar_dipan_b200/libgp.so and the CLI eshwar_dipan_b200/gp_microsim.
The CUDA sources are compiled for sm_100a only, with FMA contraction off
(--fmad=false) so that the FP64 step is bit-identical to the reference's
C arithmetic; the host C files likewise use -ffp-contract=off.
"""
import concurrent.futures
import os
import shlex
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(ROOT, "_build")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CC = os.environ.get("CC", "gcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
INC = ["-I" + os.path.join(ROOT, "include"), "-I" + CSRC]

HOST_C = ["gp_host.c", "gp_host_io.c"]
# (file, extra nvcc flags): the FP64 unit stays without FMA contraction so the
# plain step is bit-identical to the reference; the FP32 storage form may fuse.
CUDA = [("gp_device.cu", ["--fmad=false"]), ("gp_batch32.cu", ["--fmad=true"]),
        ("gp_adjoint.cu", ["--fmad=false"])]


def _run(cmd, verbose):
    if verbose:
        print(" ".join(shlex.quote(c) for c in cmd), flush=True)
    r = subprocess.run(cmd, capture_output=not verbose, text=True)
    if r.returncode != 0:
        if not verbose:
            sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("build step failed: " + " ".join(cmd[:3]))
    return r


def _stale(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False, ptxas_info=False):
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(ROOT, "include", "gp.h")] + [
        os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    objs = []
    for f in HOST_C:
        src, obj = os.path.join(CSRC, f), os.path.join(BUILD, f + ".o")
        if _stale(obj, [src] + headers):
            _run([CC, "-O2", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-std=gnu11", "-Wall",
                  "-Wno-unused-function", *INC, "-c", src, "-o", obj], verbose)
        objs.append(obj)
    jobs = []
    for f, flags in CUDA:
        src, obj = os.path.join(CSRC, f), os.path.join(BUILD, f + ".o")
        if _stale(obj, [src] + headers) or ptxas_info:
            cmd = [NVCC, *ARCH, "-lineinfo", "-O3", *flags, "-std=c++17", "-Xcompiler", "-fPIC",
                   "-Xcompiler", "-ffp-contract=off", *INC, "-c", src, "-o", obj]
            if ptxas_info:
                cmd.insert(1, "-Xptxas=-v")
            jobs.append(cmd)
        objs.append(obj)
    # the CUDA translation units are independent: compile them side by side
    with concurrent.futures.ThreadPoolExecutor(max_workers=max(1, len(jobs))) as pool:
        for r in pool.map(lambda c: _run(c, verbose), jobs):
            if ptxas_info and r.stderr:
                sys.stderr.write(r.stderr)
    lib = os.path.join(HERE, "libgp.so")
    if _stale(lib, objs):
        _run([NVCC, *ARCH, "-shared", "-cudart", "static", "-o", lib, *objs, "-lm"], verbose)
    cli_src = os.path.join(CSRC, "gp_main.c")
    cli = os.path.join(HERE, "gp_microsim")
    if os.path.exists(cli_src) and _stale(cli, [cli_src, lib] + headers):
        _run([CC, "-O2", "-ffp-contract=off", "-std=gnu11", "-Wall", *INC, cli_src, "-o", cli,
              "-L" + HERE, "-lgp", "-Wl,-rpath,$ORIGIN", "-lm"], verbose)
    return lib


if __name__ == "__main__":
    build(verbose="--verbose" in sys.argv, ptxas_info="--ptxas" in sys.argv)
    print("built", os.path.join(HERE, "libgp.so"))
