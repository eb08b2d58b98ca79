"""The reference's object API (threebodymdalgorithms_b200.simulation) over the CUDA path, used the way
the reference's own tests use its classes (src/tests/tests.cpp): build a Simulation, Init, call
GetAlgorithm().SimulationStep() or Start(), and read the counts and the particles back.  Results are
checked against the golden fixtures written by the reference itself (tests/golden/make_golden.py).
"""
import math

import numpy as np
import pytest

from tests import golden_io as GIO
from threebodymdalgorithms_b200 import csvio
from threebodymdalgorithms_b200.simulation import AUTA, NATA, P3BCA, AxilrodTeller, Simulation

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def make(algorithm, inp, iterations, meta, precision="fp64", csv_output=""):
    sim = Simulation(iterations, algorithm, AxilrodTeller(meta["nu"]), inp, meta["dt"], meta["g"], csv_output,
                     precision=precision)
    sim.Init()
    return sim


@pytest.mark.parametrize("algorithm", [NATA, AUTA])
def test_num_particle_interactions(algorithm):
    """tests.cpp:530-568: one SimulationStep evaluates all C(N,3) triplets of the N=1000 fixture."""
    inp, out, _, meta = GIO.load("tests_fixture_n1000_auta")
    sim = make(algorithm(), inp, 0, meta)
    n = len(sim.GetAllParticles()["x"])
    buffers, triplets = sim.GetAlgorithm().SimulationStep()
    assert triplets == math.comb(n, 3) == 166167000 and buffers == 1
    # the forces of that evaluation are the reference's
    st = sim.GetDecomposition().GetMyParticles()
    f = np.stack([st["fx"], st["fy"], st["fz"]], 1)
    fr = np.stack([out["fx"], out["fy"], out["fz"]], 1)
    assert rel_l2(f, fr) <= 1e-12


def test_decomposition_with_step():
    """tests.cpp:416-433: a step keeps every particle."""
    inp, _, _, meta = GIO.load("nata_n256_3steps")
    sim = make(NATA(), inp, 1, meta)
    before = sim.GetDecomposition().GetNumOfMyParticles()
    sim.Start()
    assert sim.GetDecomposition().GetNumOfMyParticles() == before == 256


@pytest.mark.parametrize("name,cls", [("p3bca_n512_c2_3steps", P3BCA), ("nata_n256_3steps", NATA),
                                      ("auta_n300_light_3steps", AUTA)])
def test_start_matches_reference_run(name, cls, tmp_path):
    """Start() over several steps: per-step counts (GetNumParticleInteractions) equal the reference's,
    the final state is within the multi-step FP64 tolerance, and with csvOutput one file per step is
    written in the reference's format."""
    inp, out, counts, meta = GIO.load(name)
    alg = cls(meta["cutoff"]) if cls is P3BCA else cls()
    base = str(tmp_path / "out.csv")
    sim = make(alg, inp, meta["iters"], meta, csv_output=base)
    sim.Start()
    got = [sim.GetNumParticleInteractions(i) for i in range(meta["iters"])]
    assert got == [int(c) for c in counts]
    assert all(sim.GetNumBufferInteractions(i) == 1 for i in range(meta["iters"]))
    st = sim.GetDecomposition().GetMyParticles()
    for k in ("x", "y", "z", "vx", "vy", "vz"):
        assert rel_l2(st[k], out[k]) <= 1e-10, k
    for i in range(meta["iters"]):
        assert (tmp_path / f"out_{i}.csv").exists()
    last = csvio.read_particles(str(tmp_path / f"out_{meta['iters'] - 1}.csv"))
    order = np.argsort(out["id"])
    assert np.allclose(last["x"], out["x"][order], rtol=1e-5, atol=1e-6)


def test_set_my_particles_then_step():
    """SetMyParticles replaces the state, as DomainDecomposition::SetMyParticles does."""
    inp, out, counts, meta = GIO.load("p3bca_n512_c2_3steps")
    sim = make(P3BCA(meta["cutoff"]), GIO.load("p3bca_n1000_c1.5_2steps")[0], 1, meta, precision="mixed")
    sim.GetDecomposition().SetMyParticles(inp)
    sim.Start()
    assert sim.GetNumParticleInteractions(0) == int(counts[0])
