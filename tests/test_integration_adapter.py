"""The C++ adapter of the integration notes (their section 2: GpuSimulation, a drop-in for the
reference's Simulation::Init + Start + GetNumParticleInteractions, src/simulation/Simulation.cpp:3-96)
compiles against the reference's own Utility::Particle (src/utility/structs.hpp:11-30, with the
oracle's stand-in mpi.h and Eigen/Dense) and links against libtbmd, so the documented binding keeps
up with include/tbmd.h.  Compile and link only, no GPU: skipped where the reference sources or the
built library are absent."""
import re
import shutil
import subprocess
from pathlib import Path

import pytest

from oracle import oracle as O

ROOT = Path(__file__).resolve().parents[1]
PKG = ROOT / "threebodymdalgorithms_b200"

DEMO = r"""
#include <cstdio>
#include "gpu_simulation.hpp"

int main(int argc, char **argv)
{
    std::vector<Utility::Particle> particles;
    for (int i = 0; i < 64; ++i)
        particles.emplace_back(i, 0.37 * (i % 4), 0.41 * ((i / 4) % 4), 0.43 * (i / 16), 0, 0, 0, 0, 0, 0, 1.0);
    if (argc < 2) return 0;  // built to be linked, run only when asked
    GpuSimulation sim(TBMD_P3BCA, particles, 2, 1e-3, 0.0, -9.81, 0.0, 2.0);
    sim.Start();
    std::printf("%llu %llu %.17g\n", (unsigned long long)sim.GetNumParticleInteractions(0),
                (unsigned long long)sim.GetNumParticleInteractions(1), particles[5].pY);
    return 0;
}
"""


def adapter_source() -> str:
    text = (ROOT / "INTEGRATION.md").read_text()
    sec = text[text.index("## 2."):text.index("## 3.")]
    m = re.search(r"```cpp\n(.*?)```", sec, re.S)
    assert m, "no C++ block in section 2 of the integration notes"
    return m.group(1)


def test_adapter_block_is_present():
    src = adapter_source()
    for name in ("class GpuSimulation", "tbmd_create", "tbmd_set_particles", "tbmd_step", "tbmd_get_particles",
                 "GetNumParticleInteractions"):
        assert name in src, name


@pytest.mark.skipif(not (O.REFERENCE_ROOT / "src" / "utility" / "structs.hpp").is_file(),
                    reason="reference sources not present")
@pytest.mark.skipif(not (PKG / "libtbmd.so").is_file(), reason="libtbmd.so not built")
@pytest.mark.skipif(shutil.which("g++") is None, reason="no g++")
def test_adapter_compiles_against_the_reference_headers(tmp_path):
    (tmp_path / "gpu_simulation.hpp").write_text("#pragma once\n" + adapter_source())
    (tmp_path / "demo.cpp").write_text(DEMO)
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", f"-I{tmp_path}", f"-I{ROOT / 'include'}",
           f"-I{O.REFERENCE_ROOT / 'src'}", f"-I{O.STUB_INCLUDE}", str(tmp_path / "demo.cpp"),
           f"-L{PKG}", "-ltbmd", f"-Wl,-rpath,{PKG}", "-o", str(tmp_path / "demo")]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    # linked against the library's exports; running without arguments touches no device
    assert subprocess.run([str(tmp_path / "demo")], timeout=60).returncode == 0
