"""Builds the B200 BigWhoop libraries (double and single precision) for sm_100a.

    python -m bigwhoop_b200.build [--jobs N] [--force]

Outputs bigwhoop_b200/lib/{double,single}/libbwc.so: the drop-in libbwc (bwc.h API plus the
bwc_b200.h extensions) with the CUDA runtime linked statically.  Objects go to
bigwhoop_b200/lib/obj/; a file is recompiled when it or any header is newer than its object.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "lib")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CUDA_INC = "/usr/local/cuda/include"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
PRECISIONS = {"double": [], "single": ["-DBWC_SINGLE_PRECISION"]}


def _sources():
    host = sorted(glob.glob(os.path.join(CSRC, "host", "*.cpp"))) + [_rate_model_source()]
    dev = sorted(glob.glob(os.path.join(CSRC, "kernels", "*.cu")))
    return host, dev


MODEL = os.path.join(HERE, "data", "pcrd_mlp.npy")


def _rate_model_source():
    """Generated C++ source holding the trained rate-control model (data/pcrd_mlp.npy, made by
    bigwhoop_b200/ratemodel.py) as the library's built-in warm-start model; a library built
    without the file has none."""
    out = os.path.join(LIB, "gen", "rate_model_data.cpp")
    os.makedirs(os.path.dirname(out), exist_ok=True)
    if os.path.exists(MODEL):
        import numpy as np
        w = np.load(MODEL).astype(np.float32).ravel()
        body = ",\n".join(", ".join(f"{float(v)!r}f" if np.isfinite(v) else "0.0f" for v in w[i:i + 8])
                           for i in range(0, w.size, 8))
        text = ("// generated by bigwhoop_b200/build.py from data/pcrd_mlp.npy\n"
                "namespace bwcb {\n"
                f"extern const float kBuiltinRateModel[{w.size}] = {{\n{body}\n}};\n"
                f"extern const int kBuiltinRateModelSize = {w.size};\n}}\n")
    else:
        text = ("namespace bwcb {\nextern const float kBuiltinRateModel[1] = {0.0f};\n"
                "extern const int kBuiltinRateModelSize = 0;\n}\n")
    if not os.path.exists(out) or open(out).read() != text:
        open(out, "w").write(text)
    return out


def _headers():
    return (glob.glob(os.path.join(CSRC, "**", "*.hpp"), recursive=True)
            + glob.glob(os.path.join(CSRC, "**", "*.cuh"), recursive=True)
            + glob.glob(os.path.join(ROOT, "include", "*.h")))


def _compile_cmd(src, obj, prec):
    inc = ["-I", os.path.join(ROOT, "include"), "-I", CSRC, "-I", CUDA_INC]
    if src.endswith(".cu"):
        return ([NVCC, "-O3", "-std=c++17", "-lineinfo", "-fmad=false", "-Xcompiler", "-fPIC",
                 "-Xcompiler", "-ffp-contract=off", "--expt-relaxed-constexpr"] + ARCH
                + PRECISIONS[prec] + inc + ["-c", src, "-o", obj])
    return (["g++", "-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fvisibility=default"]
            + PRECISIONS[prec] + inc + ["-c", src, "-o", obj])


def _stale(obj, deps):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def build(jobs=None, force=False, precisions=("double", "single"), verbose=False):
    host, dev = _sources()
    headers = _headers()
    jobs = jobs or max(1, os.cpu_count() or 1)
    outputs = {}
    for prec in precisions:
        objdir = os.path.join(LIB, "obj", prec)
        os.makedirs(objdir, exist_ok=True)
        tasks = []
        objs = []
        for src in host + dev:
            obj = os.path.join(objdir, os.path.basename(src) + ".o")
            objs.append(obj)
            if force or _stale(obj, [src] + headers):
                tasks.append(_compile_cmd(src, obj, prec))
        with cf.ThreadPoolExecutor(jobs) as ex:
            for cmd, res in zip(tasks, ex.map(lambda c: subprocess.run(c, capture_output=True, text=True), tasks)):
                if res.returncode != 0:
                    sys.stderr.write(" ".join(cmd) + "\n" + res.stdout + res.stderr)
                    raise RuntimeError(f"compilation failed: {cmd[-3]}")
                if verbose and (res.stdout or res.stderr):
                    sys.stderr.write(res.stdout + res.stderr)
        outdir = os.path.join(LIB, prec)
        os.makedirs(outdir, exist_ok=True)
        so = os.path.join(outdir, "libbwc.so")
        if force or tasks or not os.path.exists(so):
            cmd = ([NVCC, "-shared", "-cudart", "static"] + ARCH + objs
                   + ["-o", so, "-Xlinker", "-Bsymbolic", "-lpthread"])
            res = subprocess.run(cmd, capture_output=True, text=True)
            if res.returncode != 0:
                sys.stderr.write(" ".join(cmd) + "\n" + res.stdout + res.stderr)
                raise RuntimeError("link failed")
        outputs[prec] = so
    return outputs


def build_emu(precisions=("double", "single"), force=False):
    """The host build of the tier-1 kernel bodies (csrc/emu/t1_emu.cu) for the CPU unit tests:
    lib/emu/<precision>/libt1emu.so, a separate library that libbwc.so does not link."""
    src = os.path.join(CSRC, "emu", "t1_emu.cu")
    deps = [src] + _headers()
    out = {}
    for prec in precisions:
        so = os.path.join(LIB, "emu", prec, "libt1emu.so")
        os.makedirs(os.path.dirname(so), exist_ok=True)
        if force or _stale(so, deps):
            cmd = ([NVCC, "-O2", "-std=c++20", "-shared", "-Xcompiler", "-fPIC",
                    "-Xcompiler", "-ffp-contract=off", "--expt-relaxed-constexpr"] + ARCH
                   + PRECISIONS[prec] + ["-I", os.path.join(ROOT, "include"), "-I", CSRC,
                                         "-I", CUDA_INC, src, "-o", so, "-lpthread"])
            res = subprocess.run(cmd, capture_output=True, text=True)
            if res.returncode != 0:
                sys.stderr.write(" ".join(cmd) + "\n" + res.stdout + res.stderr)
                raise RuntimeError("emu build failed")
        out[prec] = so
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    for prec, so in build(a.jobs, a.force, verbose=a.verbose).items():
        print(prec, so)
    for prec, so in build_emu(force=a.force).items():
        print("emu", prec, so)


if __name__ == "__main__":
    main()
