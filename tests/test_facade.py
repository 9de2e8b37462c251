"""The C++ plugin facade (include/behavert/BehaveRT.h): reference-shaped
flocking and schooling applications compile against the C-ABI here, and on
the GPU they run through it with identical stage-wise and fused results."""
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
LIB_DIR = ROOT / "behavert_b200"
APPS = [("flocking_facade", "flocking.cfg"), ("flocking_facade", "world_radius.cfg"), ("schooling_facade", "schooling.cfg")]


CUDA = Path("/usr/local/cuda")


def _build(name: str, out: Path, cuda: bool = False):
    cmd = ["g++", "-std=c++17", "-O2", "-I", str(ROOT / "include"), str(ROOT / "tests" / "cpp" / (name + ".cpp")),
           "-o", str(out), "-L", str(LIB_DIR), "-lbehavert_b200", "-Wl,-rpath," + str(LIB_DIR)]
    if cuda:
        cmd += ["-I", str(CUDA / "include"), "-L", str(CUDA / "lib64"), "-lcudart", "-Wl,-rpath," + str(CUDA / "lib64")]
    subprocess.run(cmd, check=True, capture_output=True, text=True)


@pytest.mark.parametrize("name,cfg", APPS)
def test_facade_application_builds(tmp_path, name, cfg):
    import behavert_b200.build as b
    b.build_library()
    assert (LIB_DIR / "libbehavert_b200.so").exists()
    _build(name, tmp_path / name)


@pytest.mark.gpu
@pytest.mark.parametrize("name,cfg", APPS)
def test_facade_stagewise_equals_fused(tmp_path, name, cfg):
    exe = tmp_path / name
    _build(name, exe)
    res = subprocess.run([str(exe), str(ROOT / "tests" / "cpp" / cfg)], capture_output=True, text=True)
    print(res.stdout, res.stderr)
    assert res.returncode == 0, res.stdout + res.stderr
    assert "stage-wise == fused: yes" in res.stdout


def test_plugin_application_builds(tmp_path):
    _build("plugin_facade", tmp_path / "plugin_facade", cuda=True)


@pytest.mark.gpu
def test_plugin_arrays_and_kernel_call(tmp_path):
    """A user plugin's own per-agent arrays (Feature::User) follow their agents
    through fused and stage-wise steps, and kernelCall runs its device work in
    stream order with the before / after hooks."""
    exe = tmp_path / "plugin_facade"
    _build("plugin_facade", exe, cuda=True)
    res = subprocess.run([str(exe), str(ROOT / "tests" / "cpp" / "flocking.cfg")], capture_output=True, text=True)
    print(res.stdout, res.stderr)
    assert res.returncode == 0, res.stdout + res.stderr
    assert "snapshot follows its agents: yes" in res.stdout


@pytest.mark.parametrize("cfg,cap,world,block", [("automatic_cap.cfg", 16, 64, 0), ("flocking.cfg", 0, 64, 0),
                                                  ("world_radius.cfg", 0, 64, 128), ("keep_density.cfg", 0, 44, 256)])
def test_configuration_mapping(tmp_path, cfg, cap, world, block):
    """The reference's key names reach the engine parameters; with
    useAutomaticMaxBodiesPerCell the per-cell cap is the reference's upper
    bound 1 + cellVolume / bodyVolume (EnvGrid3DPlugIn.h:537-562); worldRadius
    and keepDensity size the cube (EnvGrid3DPlugIn.h:421-470) in whole cells;
    customBlockSize / BlockDim set the block size.  CPU only: the engine is
    created lazily and no functionality is called."""
    exe = tmp_path / "config_facade"
    _build("config_facade", exe)
    res = subprocess.run([str(exe), str(ROOT / "tests" / "cpp" / cfg)], capture_output=True, text=True)
    assert res.returncode == 0, res.stdout + res.stderr
    fields = res.stdout.split()
    got = dict(zip(fields[0::2], fields[1::2]))
    assert int(got["maxBodiesPerCell"]) == cap
    assert int(got["numBodies"]) == (1 << 10 if cfg == "automatic_cap.cfg" else 1 << 12)
    assert float(got["worldSize"]) == world and int(got["blockSize"]) == block


def test_search_depth_other_than_one_is_refused(tmp_path):
    exe = tmp_path / "config_facade"
    _build("config_facade", exe)
    res = subprocess.run([str(exe), str(ROOT / "tests" / "cpp" / "search_depth.cfg")], capture_output=True, text=True)
    assert res.returncode != 0
    assert "searchDepth must be 1 1 1" in res.stderr


def test_cluster_application_builds(tmp_path):
    _build("cluster_facade", tmp_path / "cluster_facade")


@pytest.mark.gpu
def test_cluster_inverse_hash_and_merge(tmp_path):
    """calcInverseHash against getSortedIndex, mergeClusters against a host
    restatement of the reference's merge kernel, freezeClusters a no-op."""
    exe = tmp_path / "cluster_facade"
    _build("cluster_facade", exe)
    res = subprocess.run([str(exe), str(ROOT / "tests" / "cpp" / "flocking.cfg")], capture_output=True, text=True)
    print(res.stdout, res.stderr)
    assert res.returncode == 0, res.stdout + res.stderr
    assert "inverse hash: yes" in res.stdout and ": yes" in res.stdout.split("merged")[1]


def test_logger(tmp_path):
    """UtilityLogger through m_CommonRes.getLogger(): bounded list, printf-style
    quickLog, level and sender filters (host only)."""
    exe = tmp_path / "logger_facade"
    _build("logger_facade", exe)
    res = subprocess.run([str(exe)], capture_output=True, text=True)
    assert res.returncode == 0, res.stdout + res.stderr
    assert "Flocking>> frame 59 of demo" in res.stdout and "logger: yes" in res.stdout
