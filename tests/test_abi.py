"""CPU tests of the C-ABI boundary: the library loads without a GPU, exports
every symbol include/behavert_b200.h declares, the ctypes struct mirror has
the C layout, and calls fail loudly (no CPU fallback) when no GPU is present."""
import ctypes as C
import re
import subprocess
import sys
from pathlib import Path

import pytest

import behavert_b200 as brt
from behavert_b200 import _abi
from tests.conftest import gpu_available

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "behavert_b200.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(brt_[a-z0-9_]+)\s*\(", text)))


def test_header_and_binding_agree():
    assert set(declared_functions()) == set(_abi.EXPORTED_SYMBOLS)


def test_library_exports_every_declared_symbol():
    L = brt.lib()
    for name in declared_functions():
        assert hasattr(L, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", str(brt.LIB_PATH)], capture_output=True, text=True).stdout
    for name in declared_functions():
        assert re.search(r"\sT\s%s$" % name, out, flags=re.M), name


def test_params_struct_layout_matches_c():
    src = ROOT / "tests" / "_layout_probe.c"
    exe = ROOT / "tests" / "_layout_probe"
    fields = [f[0] for f in _abi.BrtParams._fields_]
    body = "\n".join('printf("%s %%zu\\n", offsetof(brt_params, %s));' % (f, f) for f in fields)
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "behavert_b200.h"\nint main(void){\n'
                   'printf("sizeof %%zu\\n", sizeof(brt_params));\n%s\nreturn 0;}\n' % body)
    try:
        subprocess.run(["gcc", "-I", str(ROOT / "include"), "-o", str(exe), str(src)], check=True)
        out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    finally:
        src.unlink(missing_ok=True)
        exe.unlink(missing_ok=True)
    vals = dict(line.split() for line in out if line.strip())
    assert int(vals["sizeof"]) == C.sizeof(_abi.BrtParams)
    for f in fields:
        assert int(vals[f]) == getattr(_abi.BrtParams, f).offset, f


def test_params_default_and_version():
    p = brt.params_default()
    assert p.maxNeighbors == 16 and p.commonMass == 1.0 and p.alignmentParams[2] == -2.0
    assert b"sm_100a" in brt.lib().brt_version()
    assert brt.lib().brt_error_string(_abi.BRT_ERR_TIMEOUT) == b"device wait timed out"
    assert brt.radix_sort_scratch_bytes(1 << 20, 18) > 8 * (1 << 20)


@pytest.mark.skipif(gpu_available(), reason="checks the no-GPU error path")
def test_engine_without_gpu_fails_loudly():
    p = brt.params_default()
    with pytest.raises(brt.BrtError) as ei:
        brt.Engine(p)
    assert ei.value.status == _abi.BRT_ERR_NODEVICE


def test_bad_configuration_is_rejected_before_any_gpu_work():
    # Validation happens before device use when the count check passes; without
    # a GPU the NODEVICE status wins.  Either way no call may succeed.
    p = brt.params_default()
    p.worldSize = 10.0  # not a multiple of the cell size
    with pytest.raises(brt.BrtError):
        brt.Engine(p)


def test_bad_arguments_name_the_entry_point():
    """A null engine or a bad memory kind is refused before any GPU work, and
    brt_last_error names the entry point that refused it."""
    L = _abi.lib()
    cases = [("brt_step", lambda: L.brt_step(None, 0.1, 1)),
             ("brt_set_state", lambda: L.brt_set_state(None, None, None, None, None, _abi.BRT_MEM_HOST)),
             ("brt_engine_add_array", lambda: L.brt_engine_add_array(None, 4, None))]
    for name, call in cases:
        assert call() == _abi.BRT_ERR_ARG
        assert L.brt_last_error().decode() == name + ": bad arguments"


def test_facade_header_compiles():
    src = ROOT / "include" / "behavert" / "BehaveRT.h"
    if not src.exists():
        pytest.skip("C++ facade header not present")
    probe = ROOT / "tests" / "_facade_probe.cpp"
    probe.write_text('#include "behavert/BehaveRT.h"\nint main(){return 0;}\n')
    try:
        subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-I", str(ROOT / "include"), str(probe)], check=True)
    finally:
        probe.unlink(missing_ok=True)


def test_oracle_params_default_equals_the_library_defaults():
    """The CPU reference arm builds its workload from the oracle's defaults so
    that it never loads the CUDA library; both sources must agree byte for byte."""
    from oracle import oracle
    a = bytes(brt.params_default())
    b = bytes(oracle.params_default())
    assert a == b


def test_reference_arm_workload_does_not_load_the_cuda_library():
    """Building config 1 with the oracle's defaults and stepping the oracle
    maps no library of the product into the process."""
    code = ("import sys; sys.path.insert(0, %r)\n"
            "from behavert_b200 import workloads\nfrom oracle import oracle\n"
            "w = workloads.large(n=4096, defaults=oracle.params_default)\n"
            "oracle.step(w.params, w.pos, w.fwd, w.acc, w.feat, dt=w.dt, want_intermediates=False)\n"
            "maps = open('/proc/self/maps').read()\n"
            "assert 'libbehavert_b200' not in maps and '_brt_torch' not in maps, 'product library loaded'\n"
            "assert 'liboracle_brt' in maps\n" % str(ROOT))
    subprocess.run([sys.executable, "-c", code], check=True, timeout=300)
