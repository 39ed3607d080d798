"""Build recipe for libcourant_b200.so (in-tree, sm_100a).

The library is the product: the CUDA engine (csrc/engine.cu) compiled by nvcc
for sm_100a and the FP64 host setup (csrc/*.cpp) compiled by g++, linked
with the static CUDA runtime into courant_b200/lib/libcourant_b200.so. The
host code is built with FP contraction off so the FP64 plan reproduces the
reference coefficients to the bit.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIBDIR = PKG / "lib"
LIB = LIBDIR / "libcourant_b200.so"
NAPI = PKG / "napi"
SHIM_LIB = LIBDIR / "libcourant_napi_core.so"   # the Node shim's call translation behind a C ABI (node-free)
INCLUDE = PKG.parent / "include"
VERSION = "20261017.0-b200"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CUDA_LIB = Path(NVCC).resolve().parent.parent / "lib64"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CXXFLAGS = ["-O2", "-std=c++17", "-fPIC", "-fvisibility=hidden", "-ffp-contract=off", "-Wall", "-Wextra",
            "-Wno-unused-parameter", f'-DCEM_VERSION="{VERSION}"', f"-I{INCLUDE}"]
NVFLAGS = ["-O3", "-std=c++17", "-lineinfo", *ARCH, "-Xcompiler", "-fPIC,-fvisibility=hidden,-ffp-contract=off",
           "-Xptxas", "-v", f'-DCEM_VERSION="{VERSION}"', f"-I{INCLUDE}"]


def _run(cmd: list[str], log) -> None:
    log.write(" ".join(cmd) + "\n")
    r = subprocess.run(cmd, capture_output=True, text=True)
    log.write(r.stdout)
    log.write(r.stderr)
    if r.returncode != 0:
        sys.stderr.write(r.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd[:3])} ...")


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cpp")) + sorted(CSRC.glob("*.cu"))


def shim_sources() -> list[Path]:
    return [NAPI / n for n in ("arena.cpp", "shim.cpp", "shim_exports.cpp", "shim_capi.cpp")]


def needs_build() -> bool:
    if not LIB.exists() or not SHIM_LIB.exists():
        return True
    ts = SHIM_LIB.stat().st_mtime
    if any(p.stat().st_mtime > ts for p in shim_sources() + list(NAPI.glob("*.hpp")) + list(NAPI.glob("*.inc"))):
        return True
    t = LIB.stat().st_mtime
    deps = sources() + [CSRC / "exports.map"] + list(CSRC.glob("*.hpp")) + list(CSRC.glob("*.cuh")) + [INCLUDE / "courant.h", Path(__file__)]
    return any(p.stat().st_mtime > t for p in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and not needs_build():
        return LIB
    obj = PKG / "_build"
    obj.mkdir(exist_ok=True)
    LIBDIR.mkdir(exist_ok=True)
    objs = []
    with open(obj / "build.log", "w") as log:
        for src in sources():
            out = obj / (src.stem + (".cu.o" if src.suffix == ".cu" else ".o"))
            if src.suffix == ".cu":
                _run([NVCC, *NVFLAGS, "-c", str(src), "-o", str(out)], log)
            else:
                # the mode solver's band loops are plain vector loops: -O3 vectorises them
                # (element-wise, no contraction: the same bits as -O2)
                extra = ["-O3"] if src.name == "mode2d.cpp" else []
                _run(["g++", *CXXFLAGS, *extra, "-c", str(src), "-o", str(out)], log)
            objs.append(str(out))
        tmp = LIB.with_suffix(".so.tmp")
        _run(["g++", "-shared", "-o", str(tmp), *objs, f"-L{CUDA_LIB}", "-lcudart_static", "-lrt", "-ldl",
              "-lpthread", "-Wl,--exclude-libs,ALL", "-Wl,-Bsymbolic",
              f"-Wl,--version-script={CSRC / 'exports.map'}"], log)
        os.replace(tmp, LIB)
        # the Node shim's translation layer (the N-API module itself builds with node-gyp: napi/binding.gyp)
        tmp = SHIM_LIB.with_suffix(".so.tmp")
        _run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-fvisibility=hidden", "-Wall", "-Wextra",
              *[str(p) for p in shim_sources()], "-ldl", "-o", str(tmp)], log)
        os.replace(tmp, SHIM_LIB)
    if verbose:
        print((obj / "build.log").read_text())
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
