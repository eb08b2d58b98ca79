"""The reference's object API over the CUDA path, for Python callers and tests.

Mirrors the names and meaning of the reference classes at one rank:
  AxilrodTeller(v)            src/potential/AxilrodTeller.hpp:7-13 (strength nu, default 1.0)
  NATA(), AUTA(), P3BCA(c)    src/algorithm/{NATA,AUTA,P3BCA}.hpp
  Simulation(iterations, algorithm, potential, particles, dt, gForce, csvOutput)
                              src/simulation/Simulation.hpp:28-31 (topology, decomposition and the MPI
                              datatype are gone: one GPU holds every particle in a device cell grid)
  Simulation.Init / Start / GetNumParticleInteractions / GetNumBufferInteractions
  Simulation.GetAlgorithm().SimulationStep() -> (numBufferInteractions, numTriplets)
  Simulation.GetDecomposition().GetMyParticles() / SetMyParticles / ResetForces
Every computation runs in libtbmd.so; nothing here computes forces.
"""
from __future__ import annotations

from . import csvio
from ._lib import Context


class AxilrodTeller:
    def __init__(self, v: float = 1.0):
        self.v = float(v)


class Algorithm:
    name = ""
    cutoff = 0.0

    def __init__(self):
        self.simulation = None

    def SimulationStep(self):
        """Forces at the current positions without integration: (1, triplets) at one rank."""
        ctx = self.simulation._ctx
        _, _, _, _, count = ctx.forces()
        return 1, int(count)


class NATA(Algorithm):
    name = "nata"


class AUTA(Algorithm):
    name = "auta"


class P3BCA(Algorithm):
    name = "p3bca"

    def __init__(self, cutoff: float):
        super().__init__()
        self.cutoff = float(cutoff)


class Decomposition:
    def __init__(self, simulation):
        self.simulation = simulation

    def GetMyParticles(self) -> dict:
        return self.simulation._ctx.get_state()

    def SetMyParticles(self, particles: dict):
        self.simulation._ctx.set_state(particles)

    def GetNumOfMyParticles(self) -> int:
        return self.simulation._ctx.n


class Simulation:
    def __init__(self, iterations, algorithm, potential, particles, dt, gForce, csvOutput="", precision="fp64",
                 device=0, use_graph=True):
        self.iterations = int(iterations)
        self.algorithm = algorithm
        self.potential = potential
        self.particles = particles
        self.dt = float(dt)
        self.gForce = tuple(float(v) for v in gForce)
        self.csvOutput = csvOutput
        self.precision = precision
        self.device = device
        self.use_graph = use_graph
        self.numInteractions = []
        self._ctx = None
        self._decomp = Decomposition(self)

    def Init(self):
        self._ctx = Context(self.algorithm.name, self.precision, self.algorithm.cutoff, self.dt, self.gForce,
                            self.potential.v, self.device, self.use_graph)
        self._ctx.set_state(self.particles)
        self.algorithm.simulation = self

    def Start(self):
        if self.csvOutput:
            for i in range(self.iterations):
                c = self._ctx.step(1)
                self.numInteractions.append((1, int(c[0])))
                csvio.write_step(csvio.step_path(self.csvOutput, i), self._ctx.get_state())
        else:
            for c in self._ctx.step(self.iterations):
                self.numInteractions.append((1, int(c)))

    def GetAlgorithm(self):
        return self.algorithm

    def GetPotential(self):
        return self.potential

    def GetDecomposition(self):
        return self._decomp

    def GetAllParticles(self):
        return self.particles

    def GetDeltaT(self):
        return self.dt

    def GetNumIterations(self):
        return self.iterations

    def GetGForce(self):
        return self.gForce

    def GetNumBufferInteractions(self, step):
        return self.numInteractions[step][0] if step < len(self.numInteractions) else 0

    def GetNumParticleInteractions(self, step):
        return self.numInteractions[step][1] if step < len(self.numInteractions) else 0

    def GetContext(self) -> Context:
        return self._ctx
