// Runs the GpuSimulation adapter (gpu_simulation.hpp) the way the reference's main runs Simulation:
// a vector of Utility::Particle (src/utility/structs.hpp:11-30), Init, Start, then the per-step
// triplet counts.  64 particles on a 4 x 4 x 4 lattice, P3BCA with cutoff 2, two steps of 1e-3 with
// gravity (0, -9.81, 0).  Prints the two counts and then x y z vx vy vz of every particle at %.17g,
// one particle per line, in input order.  Without arguments it only builds the particles and
// exits, touching no device.
#include <cstdio>

#include "gpu_simulation.hpp"

int main(int argc, char **argv)
{
    std::vector<Utility::Particle> particles;
    for (int i = 0; i < 64; ++i)
        particles.emplace_back(i, 0.37 * (i % 4), 0.41 * ((i / 4) % 4), 0.43 * (i / 16), 0, 0, 0, 0, 0, 0, 1.0);
    if (argc < 2) return 0;
    GpuSimulation sim(TBMD_P3BCA, particles, 2, 1e-3, 0.0, -9.81, 0.0, 2.0, argv[1][0] == 'm');
    sim.Start();
    std::printf("%llu %llu\n", (unsigned long long)sim.GetNumParticleInteractions(0),
                (unsigned long long)sim.GetNumParticleInteractions(1));
    for (const Utility::Particle &p : particles)
        std::printf("%.17g %.17g %.17g %.17g %.17g %.17g\n", p.pX, p.pY, p.pZ, p.vX, p.vY, p.vZ);
    return 0;
}
