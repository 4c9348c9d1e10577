"""Build recipe for the native library (CUDA sm_100a + host C++) and the oracle checker.

``build_library()`` compiles ``csrc/`` into ``sprout_b200/libsprout_b200.so`` with nvcc for
sm_100a only.  ``build_oracle()`` compiles the C restatement in ``oracle/`` (test
infrastructure) and, when the reference sources are present on this machine, the reference
itself into ``oracle/_ref`` through ``oracle/Makefile``.
"""

from __future__ import annotations

import os
import pathlib
import shutil
import subprocess
import sys

PACKAGE = pathlib.Path(__file__).resolve().parent
ROOT = PACKAGE.parent
CSRC = PACKAGE / "csrc"
LIBRARY = PACKAGE / "libsprout_b200.so"
ORACLE = ROOT / "oracle"
ORACLE_LIB = ORACLE / "libcast_oracle.so"
REFERENCE = pathlib.Path(os.environ.get("SPROUT_REFERENCE", "/root/reference"))

SOURCES = ["common.cpp", "synth.cpp", "bvh8.cpp", "ggx_table.cpp", "light_tree.cpp", "postprocess.cpp", "image_io.cpp",
           "cast.cu",
           "guide.cu", "render.cu", "capi.cpp"]
HEADERS = ["common.hpp", "bvh8.hpp", "traverse.cuh", "material.cuh", "render.hpp", "json.hpp", "ggx_table.hpp",
           "light_tree.hpp", "guide.cuh", "guide_mlp.cuh", "guide.hpp", "tuner.hpp", "postprocess.hpp", "image_io.hpp",
           "spectral.cuh"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo",
    "-O3",
    "-std=c++17",
    "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC,-O3,-ffp-contract=off,-fvisibility=hidden,-pthread",
]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and pathlib.Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the sm_100a library cannot be built")


def _stale(target: pathlib.Path, inputs) -> bool:
    if not target.exists():
        return True
    mtime = target.stat().st_mtime
    return any(pathlib.Path(p).stat().st_mtime > mtime for p in inputs)


def build_library(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> pathlib.Path:
    inputs = [CSRC / s for s in SOURCES] + [CSRC / h for h in HEADERS] + [ROOT / "include" / "sprout_b200.h", ROOT / "include" / "sprout.h"]
    if not force and not _stale(LIBRARY, inputs):
        return LIBRARY
    cmd = [_nvcc(), "-shared", "-o", str(LIBRARY)] + [str(CSRC / s) for s in SOURCES] + NVCC_FLAGS + ["-lz"]
    if ptxas_info:
        cmd += ["-Xptxas", "-v"]
    tmp = LIBRARY.with_suffix(".so.tmp")
    cmd[cmd.index(str(LIBRARY))] = str(tmp)
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed:\n{res.stdout}\n{res.stderr}")
    if verbose or ptxas_info:
        sys.stderr.write(res.stderr)
    tmp.replace(LIBRARY)
    return LIBRARY


def build_oracle(force: bool = False, verbose: bool = False) -> pathlib.Path:
    """Compile the CPU restatement; also the reference build when its sources are here."""
    srcs = [ORACLE / "cast_oracle.c", ORACLE / "synth_oracle.c", ORACLE / "spectral_oracle.c"]
    if force or _stale(ORACLE_LIB, srcs):
        cmd = ["gcc", "-O2", "-ffp-contract=off", "-fPIC", "-shared", "-pthread"] + [str(s) for s in srcs] + [
               "-o", str(ORACLE_LIB), "-lm"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"oracle build failed:\n{res.stderr}")
    if (REFERENCE / "source").is_dir():
        jobs = str(max(1, os.cpu_count() or 1))
        res = subprocess.run(["make", "-C", str(ORACLE), f"REF={REFERENCE}", "-j", jobs],
                             capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"reference build failed:\n{res.stdout[-4000:]}\n{res.stderr[-4000:]}")
        if verbose:
            print(res.stdout[-2000:], file=sys.stderr)
    return ORACLE_LIB


if __name__ == "__main__":
    build_library(force="--force" in sys.argv, verbose=True, ptxas_info="--ptxas" in sys.argv)
    build_oracle(force="--force" in sys.argv, verbose=True)
    print(LIBRARY)
