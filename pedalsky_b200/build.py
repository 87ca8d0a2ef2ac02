"""Build libpsclouds.so (the CUDA kernels + C ABI) in-tree for sm_100a.

Usage: python -m pedalsky_b200.build [--verbose]

Each translation unit is compiled separately so per-file flags apply
(noise_bake.cu needs -fmad=false for byte-exact bakes), then linked into one
shared library next to this file.  The library carries the SHA-256 of the
sources and flags it was built from (`psc_build_id`), also written beside
it; a build is redone whenever that hash differs from the current sources',
so a library copied from elsewhere is never used for other sources, and a
copied tree (another directory, other file times) keeps its built library.
"""
from __future__ import annotations

import hashlib
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
ROOT = HERE.parent
LIB = HERE / "libpsclouds.so"
LIB_ID = HERE / "libpsclouds.so.id"
BUILD_DIR = HERE / "_build"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I", str(ROOT / "include")]
CUDA_UNITS = {
    "march.cu": [],
    "march_fast.cu": ["-prec-div=false", "-prec-sqrt=false", "-ftz=true"],
    "march_batch.cu": ["-prec-div=false", "-prec-sqrt=false", "-ftz=true"],
    "march_noalloc.cu": [],
    "grid_march.cu": ["-prec-div=false", "-prec-sqrt=false"],
    "grid_layer_grad.cu": ["-prec-div=false", "-prec-sqrt=false"],
    "march_param_grad.cu": [],
    "noise_bake.cu": ["-fmad=false"],
    "atmosphere.cu": [],
    "fetch_peak.cu": [],
    "post.cu": [],
}
CXX_UNITS = ["psc_host.cpp"]


def _host_cxx() -> str:
    for cand in ("g++-13", "g++"):
        path = shutil.which(cand)
        if path:
            return path
    raise RuntimeError("no host C++ compiler found")


def _nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(path).exists():
        raise RuntimeError("nvcc not found")
    return path


def _sources() -> list[Path]:
    return sorted(CSRC.glob("*")) + [ROOT / "include" / "psclouds.h"]


def source_hash() -> str:
    """SHA-256 over the sources (path and bytes) and the compile flags."""
    h = hashlib.sha256()
    for p in _sources():
        if p.is_file() and p.suffix in (".cu", ".cuh", ".cpp", ".h"):
            h.update(str(p.relative_to(ROOT)).encode() + b"\0" + p.read_bytes() + b"\0")
    # the include directory enters by its place in the tree, not this
    # machine's absolute path, so a copied tree keeps its hash
    flags = [f if f != str(ROOT / "include") else "include" for f in NVCC_COMMON]
    h.update(repr((ARCH, flags, sorted(CUDA_UNITS.items()), CXX_UNITS)).encode())
    return h.hexdigest()


def needs_build() -> bool:
    if not LIB.exists() or not LIB_ID.exists():
        return True
    return LIB_ID.read_text().strip() != source_hash()


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd[:3])} ... ({res.returncode})")
    if verbose and (res.stdout or res.stderr):
        sys.stderr.write(res.stdout + res.stderr)


def build(verbose: bool = False, force: bool = False, ptxas_info: bool = False) -> Path:
    if not force and not needs_build():
        return LIB
    BUILD_DIR.mkdir(exist_ok=True)
    build_id = source_hash()
    nvcc, cxx = _nvcc(), _host_cxx()
    env_ccbin = ["-ccbin", cxx]
    cmds, objs = [], []
    for unit, extra in CUDA_UNITS.items():
        obj = BUILD_DIR / (unit + ".o")
        cmd = [nvcc, *env_ccbin, *ARCH, *NVCC_COMMON, *extra, "-c", str(CSRC / unit), "-o", str(obj)]
        if ptxas_info:
            cmd += ["-Xptxas", "-v"]
        cmds.append(cmd)
        objs.append(obj)
    cuda_inc = Path(nvcc).resolve().parent.parent / "include"
    for unit in CXX_UNITS:
        obj = BUILD_DIR / (unit + ".o")
        cmds.append([cxx, "-O2", "-std=c++17", "-fPIC", "-Wall", "-Wextra", "-I", str(ROOT / "include"),
                     "-I", str(cuda_inc), f'-DPSC_BUILD_ID="{build_id}"', "-c", str(CSRC / unit), "-o",
                     str(obj)])
        objs.append(obj)
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=min(len(cmds), os.cpu_count() or 1)) as ex:
        for f in [ex.submit(_run, cmd, verbose or ptxas_info) for cmd in cmds]:
            f.result()
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc, *env_ccbin, *ARCH, "-shared", "-o", str(tmp), *map(str, objs), "-cudart", "static"]
    _run(cmd, verbose)
    os.replace(tmp, LIB)
    LIB_ID.write_text(build_id + "\n")
    return LIB


if __name__ == "__main__":
    build(verbose="--verbose" in sys.argv, force="--force" in sys.argv,
          ptxas_info="--ptxas" in sys.argv)
    print(LIB)
