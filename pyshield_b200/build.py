"""Build libshield_mp.so in place with nvcc for sm_100a.

    python -m pyshield_b200.build [--jobs N]

The plain FP64 translation unit is compiled with ``-fmad=false`` (every
multiply and add rounds separately, as in the reference's numpy
expressions); host code with ``-ffp-contract=off``. The mixed-precision unit
is compiled with ``-use_fast_math``, which changes its FP32 arithmetic only.
"""

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libshield_mp.so")
# the FP64 throughput probe bench.py uses for the step kernel's FP64 roofline
# (not part of the C-ABI)
PROBE_LIB = os.path.join(HERE, "libshield_probe.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
          "--expt-relaxed-constexpr", "-I", os.path.join(os.path.dirname(HERE), "include")]

# (source, extra flags)
UNITS = [
    ("capi.cu", ["-fmad=false"]),
    ("mp_plain.cu", ["-fmad=false"]),
    # the mixed form's FP32 process rates use the hardware's approximate
    # exp2 / log2 / reciprocal / square root with denormals flushed (these
    # options act on single precision only; its FP64 is unchanged)
    ("mp_mixed.cu", ["-use_fast_math"]),
    ("coupling.cu", ["-fmad=false"]),
    ("mp_vjp.cu", ["-fmad=false"]),
    ("physics.cu", ["-fmad=false"]),
    ("dwind.cu", ["-fmad=false"]),
]


def nvcc():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _compile(src, flags, verbose):
    obj = os.path.join(BUILD, src.replace(".cu", ".o"))
    cmd = [nvcc()] + ARCH + COMMON + flags + (["-Xptxas", "-v"] if verbose else []) + ["-c", os.path.join(CSRC, src), "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def _stale(objs):
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f != "peak.cu"] + [os.path.join(os.path.dirname(HERE), "include", "shield_mp.h"), __file__]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force=False, jobs=None, verbose=False):
    units = [u for u in UNITS if os.path.exists(os.path.join(CSRC, u[0]))]
    probe_src = os.path.join(CSRC, "peak.cu")
    if force or not os.path.exists(PROBE_LIB) or os.path.getmtime(probe_src) > os.path.getmtime(PROBE_LIB):
        tmp = PROBE_LIB + ".tmp"
        r = subprocess.run([nvcc()] + ARCH + COMMON + ["-shared", "-o", tmp, probe_src, "-cudart", "static"],
                           capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for peak.cu:\n{r.stdout}\n{r.stderr}")
        os.replace(tmp, PROBE_LIB)
    if not force and not _stale(units):
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    jobs = jobs or min(len(units), os.cpu_count() or 1)
    with cf.ThreadPoolExecutor(jobs) as ex:
        res = list(ex.map(lambda u: _compile(u[0], u[1], verbose), units))
    if verbose:
        for _, log in res:
            sys.stderr.write(log)
    objs = [o for o, _ in res]
    tmp = LIB + ".tmp"
    cmd = [nvcc()] + ARCH + ["-shared", "-o", tmp] + objs + ["-cudart", "static"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, jobs=a.jobs, verbose=a.verbose))
