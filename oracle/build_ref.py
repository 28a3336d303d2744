"""Build recipe for the oracle (test infrastructure, never the product).

* ``build_oracle()`` compiles the C restatement ``oracle/gcs_oracle.c`` into
  ``oracle/liboracle.so`` (no FMA contraction, no fast-math).
* ``build_ref()`` compiles the reference's own sources, where they lie (the
  directory named by the ``GCS_REFERENCE_DIR`` environment variable, else a
  checkout named ``reference`` beside this repository), into ``oracle/_ref/``
  (git-ignored, shipped with the built libraries):

  - ``libref_cuda.so``: the reference GPU engine (``cuda_engine.cu`` +
    ``karras_bvh.cuh`` + ``morton.h`` + CUB) for sm_100a, from a generated
    headless copy in ``oracle/_ref/build/`` with two edits: the GL-interop
    include and the one GL buffer-registration call are removed (no graphics
    stack), and the opening test's literal ``1.0f`` (cuda_engine.cu:143)
    becomes the device variable ``ref_theta_sq`` (default 1.0, i.e. the
    reference unchanged) so it can run at theta = 0.5;
  - ``libref_cpu.so``: the reference CPU Barnes-Hut (``engine.cpp``,
    ``gravity_aggregator.cpp`` with its hard-coded ``0.8f`` theta made the
    variable ``ref_cpu_theta``, ``generator.cpp``) with the flags of the
    reference's GCC build (-O3 -fopenmp -ffast-math), for x86-64-v3 so the
    library runs on any AVX2 host;
  - ``libref_morton.so``: ``morton.h`` compiled without fast-math.

Usage: ``python oracle/build_ref.py`` (both), or import and call.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
# the reference checkout: $GCS_REFERENCE_DIR, else ../reference beside the repository
REF = os.environ.get("GCS_REFERENCE_DIR") or os.path.join(os.path.dirname(REPO), "reference")
OUT = os.path.join(HERE, "_ref")
BUILD = os.path.join(OUT, "build")
NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed: %s\n%s\n%s" % (" ".join(cmd), r.stdout, r.stderr))


def _newer(target: str, sources: list[str]) -> bool:
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(s) <= t for s in sources if os.path.exists(s))


def build_oracle(force: bool = False) -> str:
    src = os.path.join(HERE, "gcs_oracle.c")
    hdr = os.path.join(HERE, "gcs_oracle.h")
    lib = os.path.join(HERE, "liboracle.so")
    if force or not _newer(lib, [src, hdr, __file__]):
        _run(["gcc", "-O2", "-std=c11", "-fPIC", "-shared", "-ffp-contract=off", "-fno-fast-math",
              src, "-o", lib, "-lm"])
    return lib


def build_ic(force: bool = False) -> str:
    """The seeded initial-conditions generator (the package's host-only
    ic_generator.cpp) as its own library, oracle/_ref/libic.so, so that
    bench.py's reference arm builds the benchmark scenario without loading
    the engine library (both arms step the identical particles)."""
    src = os.path.join(REPO, "galaxy-collision-simulator_b200", "csrc", "ic_generator.cpp")
    hdr = os.path.join(REPO, "include", "gcs.h")
    lib = os.path.join(OUT, "libic.so")
    if force or not _newer(lib, [src, hdr, __file__]):
        os.makedirs(OUT, exist_ok=True)
        _run(["g++", "-O3", "-std=c++17", "-fPIC", "-shared", "-pthread", "-I" + os.path.join(REPO, "include"),
              src, "-o", lib, "-Wl,--no-undefined"])
    return lib


def _edit_once(text: str, old: str, new: str, what: str) -> str:
    n = text.count(old)
    if n != 1:
        raise RuntimeError("reference edit '%s' expected 1 match, found %d" % (what, n))
    return text.replace(old, new)


def _headless_engine() -> str:
    with open(os.path.join(REF, "cuda_engine.cu")) as f:
        s = f.read()
    s = _edit_once(s, "#include <cuda_gl_interop.h>\n", "", "gl include")
    s = _edit_once(s, "cudaGraphicsGLRegisterBuffer(&cuda_vbo_resource, vbo_id, cudaGraphicsRegisterFlagsNone);",
                   "(void)vbo_id;", "gl register")
    s = _edit_once(s, "width * width < dist_sq * 1.0f", "width * width < dist_sq * ref_theta_sq", "theta")
    s = _edit_once(s, '#include "karras_bvh.cuh"\n',
                   '#include "karras_bvh.cuh"\n__device__ __constant__ float ref_theta_sq = 1.0f;\n',
                   "theta decl")
    path = os.path.join(BUILD, "cuda_engine_headless.cu")
    with open(path, "w") as f:
        f.write(s)
    return path


def _theta_aggregator() -> str:
    with open(os.path.join(REF, "gravity_aggregator.cpp")) as f:
        s = f.read()
    s = _edit_once(s, "float theta_sq = 0.8f * 0.8f;", "float theta_sq = ref_cpu_theta * ref_cpu_theta;",
                   "cpu theta")
    s = _edit_once(s, '#include "gravity_aggregator.h"\n',
                   '#include "gravity_aggregator.h"\nextern float ref_cpu_theta;\n', "cpu theta decl")
    path = os.path.join(BUILD, "gravity_aggregator_theta.cpp")
    with open(path, "w") as f:
        f.write(s)
    return path


def build_ref(force: bool = False) -> dict:
    """Build oracle/_ref from the reference checkout (and libic.so); returns
    {name: path}.  Without the reference only libic.so is (re)built and the
    existing reference libraries are returned."""
    libs = {k: os.path.join(OUT, "lib%s.so" % k) for k in ("ref_cuda", "ref_cpu", "ref_morton")}
    libs["ic"] = build_ic(force)
    if not os.path.isdir(REF):
        return {k: v for k, v in libs.items() if os.path.exists(v)}
    os.makedirs(BUILD, exist_ok=True)
    ref_srcs = [os.path.join(REF, f) for f in os.listdir(REF)]

    shim = os.path.join(HERE, "ref_cuda_shim.cu")
    if force or not _newer(libs["ref_cuda"], ref_srcs + [shim, __file__]):
        _headless_engine()
        _run([NVCC, "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a",
              "-Xcompiler", "-fPIC", "-shared", "-I" + REF, "-I" + BUILD, shim,
              "-o", libs["ref_cuda"]])

    shim = os.path.join(HERE, "ref_cpu_shim.cpp")
    if force or not _newer(libs["ref_cpu"], ref_srcs + [shim, __file__]):
        agg = _theta_aggregator()
        _run(["g++", "-O3", "-std=c++17", "-fopenmp", "-ffast-math", "-march=x86-64-v3", "-fPIC",
              "-shared", "-I" + REF, os.path.join(REF, "engine.cpp"), agg,
              os.path.join(REF, "generator.cpp"), shim, "-o", libs["ref_cpu"]])

    shim = os.path.join(HERE, "ref_morton_shim.cpp")
    if force or not _newer(libs["ref_morton"], ref_srcs + [shim, __file__]):
        _run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-I" + REF, shim, "-o", libs["ref_morton"]])
    return libs


if __name__ == "__main__":
    print(build_oracle(force="--force" in sys.argv))
    print(build_ref(force="--force" in sys.argv))
