"""Builds libbehavert_b200.so (sm_100a) in-tree with nvcc.

The library is compiled with ``--fmad=false`` and IEEE division / square root
so that every float operation is one correctly rounded step in source order.
Usage: ``python -m behavert_b200.build`` (or ``__graft_entry__.build()``).
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "libbehavert_b200.so"
SOURCES = ["brt_sort.cu", "brt_kernels.cu", "brt_fused.cu", "brt_resort.cu", "brt_school.cu", "brt_cluster.cu",
           "brt_adjoint.cu", "brt_engine.cu", "brt_adjoint_host.cu"]
HEADERS = ["brt_internal.cuh", "brt_kernels.cuh", "brt_agent.cuh", "brt_engine_impl.cuh"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "--fmad=false", "-prec-div=true", "-prec-sqrt=true",
    "-Xcompiler", "-fPIC,-O2,-ffp-contract=off",
    "-shared", "-cudart", "static",
]


def _nvcc() -> str:
    cand = os.environ.get("NVCC") or "/usr/local/cuda/bin/nvcc"
    return cand if Path(cand).exists() else "nvcc"


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def build_library(force: bool = False, verbose: bool = False) -> Path:
    """Compiles every source to an object in parallel (each translation unit
    is self-contained: no device code crosses files), then links."""
    deps = [CSRC / s for s in SOURCES] + [CSRC / h for h in HEADERS] + [ROOT / "include" / "behavert_b200.h", Path(__file__)]
    if not force and not _stale(LIB, deps):
        return LIB
    import concurrent.futures as cf
    import tempfile
    compile_flags = [f for f in NVCC_FLAGS if f not in ("-shared",)]
    with tempfile.TemporaryDirectory(prefix="brt_build_") as tmp:
        def compile_one(src):
            obj = Path(tmp) / (src + ".o")
            cmd = [_nvcc(), *compile_flags, "-I", str(ROOT / "include"), "-c", "-o", str(obj), str(CSRC / src)]
            if verbose:
                cmd.insert(1, "-Xptxas=-v")
            return obj, subprocess.run(cmd, capture_output=True, text=True)
        workers = max(1, min(len(SOURCES), os.cpu_count() or 1))
        with cf.ThreadPoolExecutor(workers) as ex:
            results = list(ex.map(compile_one, SOURCES))
        for _, res in results:
            if res.returncode != 0:
                sys.stderr.write(res.stdout + res.stderr)
                raise RuntimeError("nvcc failed building libbehavert_b200.so")
            if verbose:
                sys.stderr.write(res.stderr)
        link = [_nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-cudart", "static",
                "-Xcompiler", "-fPIC", "-o", str(LIB), *[str(o) for o, _ in results]]
        res = subprocess.run(link, capture_output=True, text=True)
        if res.returncode != 0:
            sys.stderr.write(res.stdout + res.stderr)
            raise RuntimeError("linking libbehavert_b200.so failed")
    return LIB


def torch_ext_path() -> Path:
    import sysconfig
    return PKG / ("_brt_torch" + sysconfig.get_config_var("EXT_SUFFIX"))


def build_torch_ext(force: bool = False) -> Path:
    """Builds the libtorch autograd binding (csrc/torch_adjoint.cpp) in-tree,
    linked against libbehavert_b200.so and the installed torch."""
    import sysconfig
    import torch
    from torch.utils import cpp_extension as ce
    target = torch_ext_path()
    src = CSRC / "torch_adjoint.cpp"
    deps = [src, ROOT / "include" / "behavert_b200.h", LIB, Path(__file__)]
    if not force and not _stale(target, deps):
        return target
    abi = int(torch.compiled_with_cxx11_abi())
    cmd = ["g++", "-shared", "-fPIC", "-O2", "-std=c++17", str(src), "-o", str(target),
           "-DTORCH_EXTENSION_NAME=_brt_torch", "-DTORCH_API_INCLUDE_EXTENSION_H", f"-D_GLIBCXX_USE_CXX11_ABI={abi}",
           "-I", sysconfig.get_paths()["include"], "-I", "/usr/local/cuda/include"]
    for inc in ce.include_paths():
        cmd += ["-isystem", inc]
    for libdir in ce.library_paths():
        cmd += ["-L", libdir, f"-Wl,-rpath,{libdir}"]
    cmd += ["-lc10", "-lc10_cuda", "-ltorch", "-ltorch_cpu", "-ltorch_python",
            "-L", str(PKG), "-lbehavert_b200", "-Wl,-rpath,$ORIGIN"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("building the torch extension failed")
    return target


def build_oracle(force: bool = False) -> Path:
    """Builds the CPU oracle (test infrastructure) under oracle/_build/."""
    target = ROOT / "oracle" / "_build" / "liboracle_brt.so"
    deps = [ROOT / "oracle" / "brt_oracle.cpp", ROOT / "oracle" / "brt_oracle_adjoint.cpp",
            ROOT / "include" / "behavert_b200.h"]
    if not force and not _stale(target, deps):
        return target
    res = subprocess.run(["make", "-C", str(ROOT / "oracle")], capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("building the oracle failed")
    return target


if __name__ == "__main__":
    build_library(force="--force" in sys.argv, verbose="-v" in sys.argv)
    build_torch_ext(force="--force" in sys.argv)
    build_oracle(force="--force" in sys.argv)
    print(LIB)
