"""The C++ adapter of the integration notes, tests/adapter/gpu_simulation.hpp (GpuSimulation, a drop-in
for the reference's Simulation::Init + Start + GetNumParticleInteractions, src/simulation/Simulation.cpp:3-96).

- Without a GPU: it compiles against the reference's own Utility::Particle (src/utility/structs.hpp:11-30,
  with the oracle's stand-in mpi.h and Eigen/Dense) and links against libtbmd, so the documented binding
  keeps up with include/tbmd.h.  Skipped where the reference sources or the built library are absent.
- On a GPU: the demo program built from it (oracle/_ref/adapter_demo, made by oracle/Makefile.ref where the
  reference's headers are) runs two P3BCA steps; its step counts and final particles must equal the
  oracle's step loop on the same particles.
"""
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O

ROOT = Path(__file__).resolve().parents[1]
PKG = ROOT / "threebodymdalgorithms_b200"
ADAPTER = ROOT / "tests" / "adapter"
DEMO_BIN = O.REF_DIR / "adapter_demo"


def test_adapter_source_is_complete():
    src = (ADAPTER / "gpu_simulation.hpp").read_text()
    for name in ("class GpuSimulation", "tbmd_create", "tbmd_set_particles", "tbmd_step", "tbmd_get_particles",
                 "GetNumParticleInteractions"):
        assert name in src, name


@pytest.mark.skipif(not (O.REFERENCE_ROOT / "src" / "utility" / "structs.hpp").is_file(),
                    reason="reference sources not present")
@pytest.mark.skipif(not (PKG / "libtbmd.so").is_file(), reason="libtbmd.so not built")
@pytest.mark.skipif(shutil.which("g++") is None, reason="no g++")
def test_adapter_compiles_against_the_reference_headers(tmp_path):
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", f"-I{ADAPTER}", f"-I{ROOT / 'include'}",
           f"-I{O.REFERENCE_ROOT / 'src'}", f"-I{O.STUB_INCLUDE}", str(ADAPTER / "demo.cpp"),
           f"-L{PKG}", "-ltbmd", f"-Wl,-rpath,{PKG}", "-o", str(tmp_path / "demo")]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    # linked against the library's exports; running without arguments touches no device
    assert subprocess.run([str(tmp_path / "demo")], timeout=60).returncode == 0


def demo_particles():
    """The 64 particles demo.cpp builds (ID, position on a 4 x 4 x 4 lattice, at rest, mass 1)."""
    i = np.arange(64)
    st = {"x": 0.37 * (i % 4), "y": 0.41 * ((i // 4) % 4), "z": 0.43 * (i // 16), "m": np.ones(64)}
    for k in ("vx", "vy", "vz", "ax", "ay", "az"):
        st[k] = np.zeros(64)
    return st


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_adapter_runs_like_the_reference(precision):
    if not DEMO_BIN.exists():
        pytest.skip("oracle/_ref/adapter_demo not built (needs the reference's headers where it is built)")
    r = subprocess.run([str(DEMO_BIN), precision], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = r.stdout.strip().splitlines()
    counts = [int(v) for v in lines[0].split()]
    got = np.array([[float(v) for v in l.split()] for l in lines[1:]])
    ref, rc = O.simulate("p3bca", 2, demo_particles(), 1e-3, (0.0, -9.81, 0.0), cutoff=2.0, nthreads=1)
    assert counts == [int(c) for c in rc]
    want = np.stack([ref[k] for k in ("x", "y", "z", "vx", "vy", "vz")], 1)
    tol = 1e-10 if precision == "fp64" else 1e-4
    assert np.linalg.norm(got[:, :3] - want[:, :3]) <= tol * np.linalg.norm(want[:, :3])
    assert np.linalg.norm(got[:, 3:] - want[:, 3:]) <= (1e-10 if precision == "fp64" else 1e-2) * \
        np.linalg.norm(want[:, 3:])
