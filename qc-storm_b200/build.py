#!/usr/bin/env python3
"""Build lib/libqcstorm_b200.so (sm_100a) from csrc/ with nvcc.

Device code is compiled with nvcc's defaults for floating point (contraction
on, IEEE division and square root, no flush-to-zero): the settings the
reference's CUDA was built with (bfgsMLE_dll.vcxproj:147-148 sets no
fast-math), which the bit-level parity of the fit kernels depends on.

Usage: python qc-storm_b200/build.py [--force] [--verbose-ptxas]
"""
import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "lib", "libqcstorm_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2,-ffp-contract=off", "-I" + INCLUDE]

UNITS = ["qcs_fit_kernels.cu", "qcs_crlb.cu", "qcs_wle.cu", "qcs_cascade.cu", "qcs_api.cu", "qcs_diag.cu", "qcs_noalloc.cu",
         "qcs_extract.cu", "qcs_post.cu", "qcs_learned.cu", "qcs_render.cu",
         "qcs_locfile.cu", "qcs_consec.cu", "qcs_stat.cu", "qcs_crlb_fisher.cu", "qcs_convnet.cu"]


def deps():
    out = []
    for d in (SRC, INCLUDE):
        for f in os.listdir(d):
            if f.endswith((".cu", ".cuh", ".h")):
                out.append(os.path.join(d, f))
    return out


def build(force=False, verbose_ptxas=False):
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    newest = max(os.path.getmtime(p) for p in deps() + [os.path.abspath(__file__)])
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) > newest:
        return LIB
    extra = ["-Xptxas", "-v"] if verbose_ptxas else []
    procs, objs = [], []
    for u in UNITS:
        o = os.path.join(BUILD, u.replace(".cu", ".o"))
        objs.append(o)
        cmd = [NVCC] + ARCH + FLAGS + extra + ["-c", os.path.join(SRC, u), "-o", o]
        procs.append((u, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    failed = False
    for u, p in procs:
        out, _ = p.communicate()
        text = out.decode(errors="replace")
        if p.returncode != 0:
            failed = True
            sys.stderr.write("nvcc failed for %s\n%s\n" % (u, text[-6000:]))
        elif verbose_ptxas:
            sys.stdout.write(text)
    if failed:
        raise RuntimeError("qcstorm_b200 build failed")
    subprocess.check_call([NVCC] + ARCH + ["-shared", "-o", LIB] + objs)
    return LIB


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose-ptxas", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.verbose_ptxas))


if __name__ == "__main__":
    main()
