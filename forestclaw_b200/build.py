"""Build recipe of libfc2d_b200.so (sm_100a), in-tree.

    python -m forestclaw_b200.build [--force]

Device code is compiled for sm_100a only.  The FP64 translation units
(k_step2_f64.cu, k_amr.cu) are compiled with -fmad=false so no FMA contraction
changes the rounding of the FP64 path; the FP32-wave unit keeps FMA.  Host C++
is compiled with -ffp-contract=off for the same reason (patch geometry, app
initial data).  The CUDA runtime is linked statically so the library loads on
any machine with a driver.
"""
from __future__ import annotations

import hashlib
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INC = os.path.join(os.path.dirname(HERE), "include")
OUT = os.path.join(HERE, "libfc2d_b200.so")
BUILD = os.path.join(HERE, "_build")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")
GXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

CU_UNITS = {
    "k_step2_f64_adv.cu": ["-fmad=false"],
    "k_step2_f64_sw.cu": ["-fmad=false"],
    "k_step2_f64_euler.cu": ["-fmad=false"],
    "k_amr.cu": ["-fmad=false"],
    "k_mass_noalloc.cu": ["-fmad=false"],
    "k_metric.cu": ["-fmad=false"],
    "k_output.cu": ["-fmad=false"],
    "k_mlp.cu": [],
    "k_mlp_tc.cu": [],
    "k_step2_f32w_adv.cu": ["--use_fast_math"],
    "k_step2_f32w_sw.cu": ["--use_fast_math"],
    "k_step2_f32w_euler.cu": ["--use_fast_math"],
}
CPP_UNITS = ["host_forest.cpp", "host_api.cpp", "apps.cpp", "host_output.cpp"]


def _sources_digest() -> str:
    h = hashlib.sha256()
    for name in sorted(os.listdir(CSRC)):
        with open(os.path.join(CSRC, name), "rb") as f:
            h.update(name.encode())
            h.update(f.read())
    with open(os.path.join(INC, "fc2d_b200.h"), "rb") as f:
        h.update(f.read())
    with open(__file__, "rb") as f:
        h.update(f.read())
    return h.hexdigest()


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError("build step failed: " + os.path.basename(cmd[-1]))
    return r


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    stamp = os.path.join(BUILD, "stamp")
    digest = _sources_digest()
    if not force and os.path.exists(OUT) and os.path.exists(stamp):
        with open(stamp) as f:
            if f.read().strip() == digest:
                return OUT
    common = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-I", CSRC, "-I", INC, "-lineinfo"]
    jobs = []   # (object, command): the units compile in parallel
    for cu, extra in CU_UNITS.items():
        obj = os.path.join(BUILD, cu + ".o")
        jobs.append((obj, [NVCC, *ARCH, *common, *extra, "-Xptxas", "-v" if verbose else "-O3", "-c",
                           os.path.join(CSRC, cu), "-o", obj]))
    for cpp in CPP_UNITS:
        obj = os.path.join(BUILD, cpp + ".o")
        jobs.append((obj, [GXX, "-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-Wall",
                           "-I", CSRC, "-I", INC, "-I", os.path.join(CUDA, "include"), "-c",
                           os.path.join(CSRC, cpp), "-o", obj]))
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        results = list(ex.map(lambda j: _run(j[1]), jobs))
    if verbose:
        for r in results:
            sys.stderr.write(r.stderr)
    objs = [j[0] for j in jobs]
    _run([NVCC, *ARCH, "-shared", "-cudart", "static", "-Xcompiler", "-fPIC", "-o", OUT, *objs])
    with open(stamp, "w") as f:
        f.write(digest)
    return OUT


USER_EXAMPLES = os.path.join(os.path.dirname(HERE), "tests", "user_solvers")


def build_user_examples(force: bool = False) -> list:
    """Compile the application-solver examples of tests/user_solvers (each .cu with its own
    __device__ solvers, registered through include/fc2d_b200_user.cuh) into lib<name>.so
    beside its source, linked against libfc2d_b200.so."""
    out = []
    if not os.path.isdir(USER_EXAMPLES):
        return out
    build(force=force)
    for name in sorted(os.listdir(USER_EXAMPLES)):
        if not name.endswith(".cu"):
            continue
        src = os.path.join(USER_EXAMPLES, name)
        so = os.path.join(USER_EXAMPLES, "lib" + name[:-3] + ".so")
        deps = [src, OUT, os.path.join(INC, "fc2d_b200_user.cuh")] + \
            [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
        if not force and os.path.exists(so) and os.path.getmtime(so) >= max(os.path.getmtime(d) for d in deps):
            out.append(so)
            continue
        _run([NVCC, *ARCH, "-std=c++17", "-O3", "-fmad=false", "-I", INC, "-I", CSRC, "-Xcompiler", "-fPIC",
              "-shared", src, "-o", so, "-L", HERE, "-lfc2d_b200", "-Xlinker", "-rpath,$ORIGIN/../../forestclaw_b200"])
        out.append(so)
    return out


if __name__ == "__main__":
    p = build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(p)
