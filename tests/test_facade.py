"""The C++ plugin facade (include/behavert/BehaveRT.h): it compiles against
the C-ABI here, and on the GPU a reference-shaped flocking application runs
through it with identical stage-wise and fused results."""
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
LIB_DIR = ROOT / "behavert_b200"


def _build(out: Path):
    cmd = ["g++", "-std=c++17", "-O2", "-I", str(ROOT / "include"), str(ROOT / "tests" / "cpp" / "flocking_facade.cpp"),
           "-o", str(out), "-L", str(LIB_DIR), "-lbehavert_b200", "-Wl,-rpath," + str(LIB_DIR)]
    subprocess.run(cmd, check=True, capture_output=True, text=True)


def test_facade_application_builds(tmp_path):
    import behavert_b200.build as b
    b.build_library()
    (LIB_DIR / "libbehavert_b200.so").exists()
    _build(tmp_path / "flocking_facade")


@pytest.mark.gpu
def test_facade_stagewise_equals_fused(tmp_path):
    exe = tmp_path / "flocking_facade"
    _build(exe)
    res = subprocess.run([str(exe), str(ROOT / "tests" / "cpp" / "flocking.cfg")], capture_output=True, text=True)
    print(res.stdout, res.stderr)
    assert res.returncode == 0, res.stdout + res.stderr
    assert "stage-wise == fused: yes" in res.stdout
