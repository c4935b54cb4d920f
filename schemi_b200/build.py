"""Build recipe of the CUDA library ``schemi_b200/lib/libschemi_fv.so`` (sm_100a).

    python -m schemi_b200.build            # or build() from Python

Translation units (compiled in parallel):
  csrc/fv_f64_ns<N>_<eos>.cu  FP64 step kernels for N species and one EOS, --fmad=false (bit-exact
                        with the reference)
  csrc/fv_f32_ns<N>_<eos>.cu  FP32-flux step kernels for N species and one EOS, fast math
  csrc/fv_dispatch.cu   selects the unit of a species count and an EOS
  csrc/fv_capi.cu       C-ABI, upload/download/finalize kernels, device time loop (--fmad=false)
  csrc/fv_batch.cu      batched ensemble (--fmad=false)
  csrc/fv_noalloc.cu    the step without device allocation (--fmad=false)
  csrc/fv_chem.cu       chemistry pass (Cl2, A+B->2C), FP64 (--fmad=false)
  csrc/fv_diffusion.cu  diffusion stage (explicit, constant coefficients), FP64 (--fmad=false)
  csrc/fv_adjoint.cu    recorded trajectories, checkpoints and the adjoint sweep
  csrc/fv_adjoint_f64.cu / fv_adjoint_f32.cu  adjoint step kernels per arithmetic
nvcc cross-compiles for sm_100a without a GPU.

The task-deck driver ``schemi_b200/lib/fvrun`` (host/fvrun.cpp, C++17, g++) links the library
through its C-ABI with an $ORIGIN rpath, so the pair can be moved together.
"""

from __future__ import annotations

import concurrent.futures as cf
import os
import re
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libschemi_fv.so")
DRIVER = os.path.join(LIBDIR, "fvrun")
DRIVER_SRC = os.path.join(HERE, "host", "fvrun.cpp")
BUILD = os.path.join(HERE, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2", "--expt-relaxed-constexpr",
          "-I", os.path.join(HERE, "..", "include")]
UNITS = {
    "fv_capi.cu": ["--fmad=false"],
    "fv_dispatch.cu": [],
    "fv_chem.cu": ["--fmad=false"],
    "fv_diffusion.cu": ["--fmad=false"],
    "fv_adjoint.cu": [],
    "fv_adjoint_f64.cu": [],
    "fv_adjoint_f32.cu": ["-use_fast_math"],
}
for _ns in (1, 2, 3, 4):
    for _eos in ("ideal", "vdw", "real"):
        UNITS[f"fv_f64_ns{_ns}_{_eos}.cu"] = ["--fmad=false"]
        UNITS[f"fv_f32_ns{_ns}_{_eos}.cu"] = ["-use_fast_math"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


_INCLUDE = re.compile(r'^\s*#\s*include\s+"([^"]+)"', re.M)


def _closure(path: str, seen=None) -> set:
    """The file and every local header it includes, directly or through other headers (quoted
    includes resolved beside the including file, then in csrc/ and include/)."""
    seen = set() if seen is None else seen
    path = os.path.normpath(path)
    if path in seen or not os.path.exists(path):
        return seen
    seen.add(path)
    with open(path, encoding="utf-8", errors="replace") as f:
        text = f.read()
    for name in _INCLUDE.findall(text):
        for base in (os.path.dirname(path), CSRC, os.path.join(HERE, "..", "include")):
            cand = os.path.join(base, name)
            if os.path.exists(cand):
                _closure(cand, seen)
                break
    return seen


def _sources():
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cuh", ".inc", ".h"))]


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False, extra_flags=None) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    units = dict(UNITS)
    if os.path.exists(os.path.join(CSRC, "fv_noalloc.cu")):
        units["fv_noalloc.cu"] = ["--fmad=false"]
    if os.path.exists(os.path.join(CSRC, "fv_batch.cu")):
        units["fv_batch.cu"] = ["--fmad=false"]
    objs = []
    jobs = []
    for unit, flags in units.items():
        obj = os.path.join(BUILD, unit.replace(".cu", ".o"))
        objs.append(obj)
        if force or _stale(obj, sorted(_closure(os.path.join(CSRC, unit)))):
            cmd = [nvcc(), *ARCH, *COMMON, *flags, *(extra_flags or []), "-c", os.path.join(CSRC, unit), "-o", obj]
            jobs.append(cmd)
    with cf.ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 4))) as ex:
        futs = [ex.submit(subprocess.run, cmd, capture_output=True, text=True) for cmd in jobs]
        for cmd, fut in zip(jobs, futs):
            res = fut.result()
            if verbose or res.returncode != 0:
                sys.stderr.write(" ".join(cmd) + "\n" + res.stdout + res.stderr)
            if res.returncode != 0:
                raise RuntimeError(f"nvcc failed for {cmd[-3]}")
    if force or jobs or _stale(LIB, objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError("link failed:\n" + res.stdout + res.stderr)
    build_driver(force=force)
    return LIB


def build_driver(force: bool = False) -> str:
    """Compile the task-deck driver against the built library."""
    deps = [DRIVER_SRC, os.path.join(HERE, "host", "deck.hpp"), LIB, os.path.join(HERE, "..", "include", "fvstep.h")]
    if force or _stale(DRIVER, deps):
        cmd = [os.environ.get("CXX", "g++"), "-std=c++17", "-O2", "-Wall", "-I", os.path.join(HERE, "..", "include"),
               DRIVER_SRC, "-o", DRIVER, "-L", LIBDIR, "-lschemi_fv", "-Wl,-rpath,$ORIGIN"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError("driver build failed:\n" + " ".join(cmd) + "\n" + res.stdout + res.stderr)
    return DRIVER


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
