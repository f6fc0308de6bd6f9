#!/usr/bin/env python3
"""TEST INFRASTRUCTURE ONLY: build the reference QC-STORM library for the host.

Compiles the reference's own CUDA sources (MLEbfgs/bfgs_MLE_dll x64/bfgsMLE_dll/
bfgsMLE_dll/) with g++ against the host shim in oracle/refshim/, links them with
oracle/ref_harness.cpp and writes oracle/_ref/libqcs_ref_host.so.  The result
runs the reference's fit kernels, WLE pre-pass, CRLB, cascade orchestration,
ROI extraction, super-resolution render, consecutive-frame merging and the
localization statistics on the CPU, one emulated CUDA block
at a time; it is the checker
the CPU oracle (oracle/qcs_oracle.c) is pinned against.

Two mechanical rewrites are applied while the sources are read, into a
temporary directory outside the repository that is deleted afterwards (no
reference source text is kept in the repository):
  1. kernel launches `k<<<cfg>>>(args)` become `qcs_emu_cfg(cfg).run((k), args)`,
     because g++ has no launch syntax;
  2. SplineInterpolation.h names a function-pointer parameter after an
     enclosing template parameter (InputDataLen), which MSVC accepts and GCC
     rejects; the parameter name is dropped (names in a function-pointer
     parameter list have no meaning);
  3. gpuRemoveBackgroundIntensity (LDROIExtraction_ImageFiltering.cu:240-250)
     has its 32 threads (one warp) read their neighbours' BkgVal entries
     after one barrier and overwrite their own entry in the next loop
     iteration before the next barrier.  A warp executing in lock step reads
     before any lane writes; the emulator runs one thread at a time between
     barriers, so lane 0 would overwrite its entry before lane 1 reads it.
     A __syncthreads() is inserted after the read, which restores the
     lock-step order on the host and changes nothing the GPU computes.
Every unit is also compiled with <cstring> included first: BFGS for curve
fitting/BFGSOptimizer.h calls memset and memcpy without including it (MSVC's
headers declare them on the way), which GCC rejects.
Nothing else is changed.  Only the built .so lands in oracle/_ref/.

With --gpu the same sources are compiled unmodified by nvcc for sm_100a
(only rewrite 2 applies) with oracle/ref_harness_gpu.cu into
oracle/_ref/libqcs_ref_gpu.so: the reference's own CUDA code, run on the
B200 as the bit-level checker of the product kernels.

Usage: python oracle/build_ref.py [--ref PATH] [--force] [--gpu]
Exits 0 without building when the reference tree is absent (GPU hosts).
"""
import argparse
import os
import re
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
# The localization library inside the reference checkout; the checkout itself
# is BASELINE.json's reference_path (or --ref names the library directory).
LIB_SUBDIR = os.path.join("MLEbfgs", "bfgs_MLE_dll x64", "bfgsMLE_dll", "bfgsMLE_dll")


def default_ref():
    """The reference's localization library, from BASELINE.json's reference_path."""
    import json
    try:
        with open(os.path.join(os.path.dirname(HERE), "BASELINE.json")) as f:
            root = json.load(f).get("reference_path")
    except (OSError, ValueError):
        root = None
    return os.path.join(root, LIB_SUBDIR) if root else None


OUT_DIR = os.path.join(HERE, "_ref")
OUT_SO = os.path.join(OUT_DIR, "libqcs_ref_host.so")
OUT_GPU_SO = os.path.join(OUT_DIR, "libqcs_ref_gpu.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

# Reference sub-directories and translation units of the localization path.
DIRS = ["bfgsMLE_Loc_LD", "bfgsMLE_Loc_HD", "bfgsMLE_Loc_top", "WLEParaEstimation",
        "SubregionExtraction", "cudaWrapper", "ImgRender", "ConsecutiveFit", "StatisticsInfo",
        "BFGS for curve fitting"]
UNITS = [
    "bfgsMLE_Loc_LD/bfgs_base.cu",
    "bfgsMLE_Loc_LD/bfgsMLE_Single_Emitter_Fit.cu",
    "bfgsMLE_Loc_HD/bfgsMLE_Multi_Emitter_Fit.cu",
    "bfgsMLE_Loc_top/bfgs_top.cu",
    "bfgsMLE_Loc_top/bfgs_top_MoleculeClasify.cu",
    "bfgsMLE_Loc_top/LocPrecCalc_GaussianCRLB.cu",
    "bfgsMLE_Loc_top/ZeroLocalizationsRemove.cu",
    "WLEParaEstimation/WLEParaEstimation.cpp",
    "WLEParaEstimation/WLEParaEstimation_core.cu",
    "SubregionExtraction/LDROIExtraction.cu",
    "SubregionExtraction/LDROIExtraction_ImageFiltering.cu",
    "SubregionExtraction/LDROIExtraction_ROIExtraction.cu",
    "ImgRender/ImageRender_2d.cu",
    "ImgRender/ImageRender_3d.cu",
    "ImgRender/ImageRender_top.cu",
    "ImgRender/ImageRerender_rc.cu",
    "ConsecutiveFit/ConsecutiveFit.cu",
    "ConsecutiveFit/ConsecutiveFit_top.cu",
    "StatisticsInfo/statisticsInfo.cu",
    "StatisticsInfo/statisticsInfo_densityCalc.cu",
    "StatisticsInfo/statisticsInfo_rc.cu",
    "StatisticsInfo/statisticsInfo_top.cu",
    "BFGS for curve fitting/CurveFitting.cpp",
]

LAUNCH = re.compile(
    r"([A-Za-z_]\w*(?:\s*<[^<>;()]*>)?)\s*<<\s*<([^;]*?)>>\s*>\s*\(\s*(\)?)")
FNPTR_PARAM = re.compile(
    r"(\(\s*\*\s*FindPositionID\s*\)\s*\([^()]*?)int\s+InputDataLen\s*,")


BKG_MEAN = re.compile(r"(float\s+MeanBkg\s*=\s*\(BkgVal\[Sel0\][^;]*;)")


def rewrite(text, launches=True):
    def launch(m):
        kernel, cfg, empty = m.group(1), m.group(2).strip(), m.group(3)
        return "qcs_emu_cfg(%s).run((%s)%s" % (cfg, kernel, ")" if empty else ", ")
    if launches:
        text, _ = LAUNCH.subn(launch, text)
        text = BKG_MEAN.sub(r"\1 __syncthreads();", text)
    text = FNPTR_PARAM.sub(r"\1int,", text)
    return text


def stage_sources(ref, tmp, launches):
    for d in DIRS:
        src = os.path.join(ref, d)
        dst = os.path.join(tmp, d)
        os.makedirs(dst, exist_ok=True)
        for name in os.listdir(src):
            if not name.endswith((".h", ".cu", ".cpp")):
                continue
            with open(os.path.join(src, name), "r", encoding="latin-1") as f:
                text = f.read()
            with open(os.path.join(dst, name), "w", encoding="latin-1") as f:
                f.write(rewrite(text, launches))


def run_parallel(cmds):
    procs = [(c, subprocess.Popen(c, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)) for c in cmds]
    ok = True
    for c, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            ok = False
            sys.stdout.write("build_ref: failed: %s\n%s\n" % (" ".join(c)[-300:], out.decode(errors="replace")[-4000:]))
    return ok


def build_gpu(args):
    if not args.ref or not os.path.isdir(args.ref):
        print("build_ref: reference tree not present, skipping")
        return 0
    ours = [os.path.join(HERE, "ref_harness_gpu.cu"), os.path.abspath(__file__),
            os.path.join(HERE, "..", "include", "qcstorm_b200.h")]
    if (not args.force and os.path.exists(OUT_GPU_SO)
            and os.path.getmtime(OUT_GPU_SO) > newest_mtime(ours)):
        print("build_ref: gpu build up to date")
        return 0
    os.makedirs(OUT_DIR, exist_ok=True)
    tmp = tempfile.mkdtemp(prefix="qcs_refsrc_")
    try:
        stage_sources(args.ref, tmp, launches=False)
        open(os.path.join(tmp, "stdafx.h"), "w").close()
        incs = ["-I" + tmp] + ["-I" + os.path.join(tmp, d) for d in DIRS]
        flags = ["-std=c++17", "-O3", "-gencode", "arch=compute_100a,code=sm_100a", "-Xcompiler", "-fPIC",
                 "-w", "-D__declspec(x)=", "-x", "cu", "-rdc=false", "--pre-include", "cstring"]
        units = [os.path.join(tmp, u) for u in UNITS] + [os.path.join(HERE, "ref_harness_gpu.cu")]
        objs, cmds = [], []
        for i, u in enumerate(units):
            o = os.path.join(tmp, "g%02d.o" % i)
            objs.append(o)
            cmds.append([NVCC] + flags + incs + ["-c", u, "-o", o])
        if not run_parallel(cmds):
            return 1
        subprocess.check_call([NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", OUT_GPU_SO] + objs)
        print("build_ref: wrote", OUT_GPU_SO)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    return 0


def newest_mtime(paths):
    return max(os.path.getmtime(p) for p in paths)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=None, help="the reference's bfgsMLE_dll library directory "
                    "(default: BASELINE.json's reference_path + " + LIB_SUBDIR + ")")
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--gpu", action="store_true")
    args = ap.parse_args()
    if args.ref is None:
        args.ref = default_ref()
    if args.gpu:
        return build_gpu(args)
    if not args.ref or not os.path.isdir(args.ref):
        print("build_ref: reference tree not present, skipping")
        return 0
    ours = [os.path.join(HERE, "ref_harness.cpp"), os.path.join(HERE, "refshim", "cuda_runtime.h"),
            os.path.join(HERE, "refshim", "simt_emu.cpp"), os.path.abspath(__file__),
            os.path.join(HERE, "..", "include", "qcstorm_b200.h")]
    if (not args.force and os.path.exists(OUT_SO)
            and os.path.getmtime(OUT_SO) > newest_mtime(ours)):
        print("build_ref: up to date")
        return 0
    os.makedirs(OUT_DIR, exist_ok=True)
    tmp = tempfile.mkdtemp(prefix="qcs_refsrc_")
    try:
        for d in DIRS:
            src = os.path.join(args.ref, d)
            dst = os.path.join(tmp, d)
            os.makedirs(dst, exist_ok=True)
            for name in os.listdir(src):
                if not name.endswith((".h", ".cu", ".cpp")):
                    continue
                with open(os.path.join(src, name), "r", encoding="latin-1") as f:
                    text = f.read()
                with open(os.path.join(dst, name), "w", encoding="latin-1") as f:
                    f.write(rewrite(text))
        incs = ["-I" + os.path.join(HERE, "refshim")] + ["-I" + os.path.join(tmp, d) for d in DIRS]
        flags = ["-std=c++17", "-O2", "-fPIC", "-ffp-contract=off", "-w", "-D__declspec(x)=", "-include", "cstring"]
        objs = []
        units = [os.path.join(tmp, u) for u in UNITS]
        units += [os.path.join(HERE, "ref_harness.cpp"), os.path.join(HERE, "refshim", "simt_emu.cpp")]
        procs = []
        for i, u in enumerate(units):
            o = os.path.join(tmp, "u%02d.o" % i)
            objs.append(o)
            cmd = ["g++", "-x", "c++"] + flags + incs + ["-c", u, "-o", o]
            procs.append((u, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
        ok = True
        for u, p in procs:
            out, _ = p.communicate()
            if p.returncode != 0:
                ok = False
                sys.stdout.write("build_ref: compile failed for %s\n%s\n" % (u, out.decode(errors="replace")[-4000:]))
        if not ok:
            return 1
        cmd = ["g++", "-shared", "-o", OUT_SO] + objs
        subprocess.check_call(cmd)
        print("build_ref: wrote", OUT_SO)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
