"""Builds libfot.so in-tree with nvcc for sm_100a.

    python -m cuda_fot_b200.build [--functor-dir DIR] [--jobs N]

Each csrc/*.cu is compiled to an object under cuda_fot_b200/_build/ (in
parallel) and linked into cuda_fot_b200/libfot.so.  Device code is compiled
with -fmad=false so that no multiply-add is fused: every FP64/FP32 operation
rounds as written, as in the reference's serial loop, which makes a coloured
run bit-identical to the CPU replay of its colour order.  The atomic
executor's units (csrc/atomic_*.cu) are the exception: they are compiled
with -fmad=true, as the reference compiles its device code, because atomic
results differ from the serial loop by summation order anyway (checked
within 1e-12 FP64 / 1e-5 FP32) and contraction cuts the instruction count
of the heavy functors.  --functor-dir
compiles the loops against another directory of *_func.hpp user functions in
the reference's drop-in format.
"""
import argparse
import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libfot.so")

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-std=c++17", "-O3", "-lineinfo", "--expt-relaxed-constexpr",
         "-Xcompiler", "-fPIC,-O2", "-diag-suppress", "177",
         "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]


def fmad_flag(src):
    """Multiply-add contraction only in the atomic executor's units."""
    return "-fmad=true" if os.path.basename(src).startswith("atomic_") else "-fmad=false"


def _compile(src, obj, extra):
    cmd = [NVCC] + ARCH + FLAGS + [fmad_flag(src)] + extra + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj


def build(functor_dir=None, jobs=None, out=LIB, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    extra = []
    tag = ""
    if functor_dir:
        extra.append(f"-DFOT_FUNCTOR_DIR={os.path.abspath(functor_dir)}")
        tag = "_alt"
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    objs = [os.path.join(BUILD, os.path.basename(s)[:-3] + tag + ".o") for s in srcs]
    headers = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.hpp")) + \
        glob.glob(os.path.join(CSRC, "kernels", "*.hpp")) + [os.path.join(ROOT, "include", "fot.h")]
    newest_hdr = max(os.path.getmtime(h) for h in headers)
    todo = []
    for s, o in zip(srcs, objs):
        if functor_dir or not os.path.exists(o) or os.path.getmtime(o) < max(os.path.getmtime(s), newest_hdr):
            todo.append((s, o))
    with cf.ThreadPoolExecutor(max_workers=jobs or os.cpu_count()) as ex:
        for o in ex.map(lambda so: _compile(so[0], so[1], extra), todo):
            if verbose:
                print("compiled", os.path.relpath(o, ROOT))
    if todo or not os.path.exists(out):
        cmd = [NVCC] + ARCH + ["-shared", "-o", out] + objs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--functor-dir")
    ap.add_argument("--jobs", type=int)
    ap.add_argument("--out", default=LIB)
    a = ap.parse_args(argv)
    print(build(a.functor_dir, a.jobs, a.out, verbose=True))


if __name__ == "__main__":
    sys.exit(main())
