"""Builds the reference's own host-compilable helpers of this path into
oracle/_ref/libbrt_ref.so (TEST INFRASTRUCTURE: the oracle's check against
the reference itself).

The reference's device functions are compiled with g++ from the files where
they lie in the BehaveRT sources (BEHAVERT_REFERENCE, default /root/reference):

  Core/common_resources.cu                      (vector and integration helpers)
  PlugIns/EnvGrid3D/envgrid3d_resources.cu      (calcGridPos, calcGridHash)
  PlugIns/Proximity3D/Proximity3D_resources.cu  (checkForNeighbor, checkForNeighborsInCell)
  PlugIns/OpenSteerWrapper/OpenSteerWrapper_resources.cu
                                                (inBoidNeighborhood, calcSeparation,
                                                 calcAlignment, calcCohesion,
                                                 applySteeringForceSingle)

with the stand-ins of oracle/ref_shim/ (CUDA keywords, the SDK vector
helpers, textures as host arrays) force-included.  The sources use MSVC
include paths with backslashes (e.g. "..\\EnvGrid3D\\envgrid3d_resources.cu");
the recipe writes one redirect header per such name into oracle/_ref/gen/,
forwarding to the real file.  Nothing of the reference is copied: every
redirect is one #include line.  oracle/ref_harness.cpp adds the C entry
points the tests call.  Outputs go to oracle/_ref/ only.

Usage: python oracle/build_ref.py   (exits 0 with a message when the
reference sources are absent, e.g. on a machine without them).
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
GEN = OUT / "gen"
LIB = OUT / "libbrt_ref.so"
REF = Path(os.environ.get("BEHAVERT_REFERENCE", "/root/reference"))

# include name as written in the reference sources -> file under REF
REDIRECTS = {
    "include\\Proximity3D_kernel.cuh": "PlugIns/Proximity3D/include/Proximity3D_kernel.cuh",
    "include\\proximity3d_kernel.cuh": "PlugIns/Proximity3D/include/Proximity3D_kernel.cuh",
    "include\\envgrid3d_kernel.cuh": "PlugIns/EnvGrid3D/include/envgrid3d_kernel.cuh",
    "include\\body3d_kernel.cuh": "PlugIns/Body/include/body3d_kernel.cuh",
    "include\\OpenSteerWrapper_kernel.cuh": "PlugIns/OpenSteerWrapper/include/OpenSteerWrapper_kernel.cuh",
    "..\\EnvGrid3D\\include\\envgrid3d_kernel.cuh": "PlugIns/EnvGrid3D/include/envgrid3d_kernel.cuh",
    "..\\EnvGrid3D\\envgrid3d_resources.cu": "PlugIns/EnvGrid3D/envgrid3d_resources.cu",
    "..\\Body\\include\\body3d_kernel.cuh": "PlugIns/Body/include/body3d_kernel.cuh",
    "..\\Body\\body3d_resources.cu": "PlugIns/Body/body3d_resources.cu",
    "..\\Proximity3D\\include\\Proximity3D_kernel.cuh": "PlugIns/Proximity3D/include/Proximity3D_kernel.cuh",
    "..\\Proximity3D\\Proximity3D_resources.cu": "PlugIns/Proximity3D/Proximity3D_resources.cu",
    "proximity3d_resources.cu": "PlugIns/Proximity3D/Proximity3D_resources.cu",
}
SOURCES = ["Core/common_resources.cu", "PlugIns/EnvGrid3D/envgrid3d_resources.cu",
           "PlugIns/Proximity3D/Proximity3D_resources.cu", "PlugIns/OpenSteerWrapper/OpenSteerWrapper_resources.cu",
           "PlugIns/Proximity3D/Proximity3D_kernel.cu", "PlugIns/OpenSteerWrapper/OpenSteerWrapper_kernel.cu"]


def available() -> bool:
    return all((REF / s).exists() for s in SOURCES)


def build(force: bool = False, verbose: bool = False) -> Path | None:
    if not available():
        if verbose:
            print("reference sources not found under %s: oracle/_ref not built" % REF)
        return None
    deps = [HERE / "ref_harness.cpp", Path(__file__)] + list((HERE / "ref_shim").glob("*"))
    if not force and LIB.exists() and all(d.stat().st_mtime <= LIB.stat().st_mtime for d in deps):
        return LIB
    GEN.mkdir(parents=True, exist_ok=True)
    for name, target in REDIRECTS.items():
        (GEN / name).write_text('#include "%s"\n' % (REF / target))
    cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-ffp-contract=off", "-fno-fast-math",
           "-w", "-include", str(HERE / "ref_shim" / "cuda_standins.h"),
           "-I", str(HERE / "ref_shim"), "-I", str(GEN), "-I", str(REF / "Core"), "-I", str(REF / "Core" / "include"),
           "-DBRT_REF_ROOT=" + str(REF),
           str(HERE / "ref_harness.cpp"), "-Wl,--no-undefined", "-o", str(LIB)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("compiling the reference helpers failed")
    return LIB


if __name__ == "__main__":
    out = build(force="--force" in sys.argv, verbose=True)
    print(out if out else "skipped")
