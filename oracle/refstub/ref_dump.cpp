// Full-precision dump driver around the reference's own classes (test infrastructure only).
//
// It wires Simulation + {NATA|AUTA|P3BCA} + AxilrodTeller(1.0) + {Ring|Cart}Topology +
// {Atom|RegularGrid}Decomposition exactly as the reference's main does for one rank
// (src/main.cpp:32-105, 516-559) and then either
//   --mode sim    : runs Simulation::Start() (src/simulation/Simulation.cpp:28-81) for the given
//                   iterations, or
//   --mode forces : calls Algorithm::SimulationStep() once at the input positions, the way the
//                   reference's tests call it (src/tests/tests.cpp:539),
// and prints every particle with %.17g plus the per-step (buffer, particle) interaction counts
// (Simulation::GetNumBufferInteractions / GetNumParticleInteractions, Simulation.cpp:89-96).
//
// usage: ref_dump --algo nata|auta|p3bca --csv FILE [--mode sim|forces] [--iters N] [--dt D]
//                 [--g GX GY GZ] [--cutoff C] [--nu NU]
#include <chrono>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "algorithm/AUTA.hpp"
#include "algorithm/NATA.hpp"
#include "algorithm/P3BCA.hpp"
#include "decomposition/AtomDecomposition.hpp"
#include "decomposition/RegularGridDecomposition.hpp"
#include "potential/AxilrodTeller.hpp"
#include "simulation/Simulation.hpp"
#include "topology/CartTopology.hpp"
#include "topology/RingTopology.hpp"

int main(int argc, char **argv)
{
    std::string algo = "auta", csv, mode = "sim";
    int iters = 1;
    double dt = 0.001, cutoff = 0.0, nu = 1.0;
    double g[3] = {0.0, 0.0, 0.0};
    for (int i = 1; i < argc; ++i) {
        std::string f = argv[i];
        auto need = [&](int k) {
            if (i + k >= argc) {
                std::fprintf(stderr, "ref_dump: %s needs %d value(s)\n", f.c_str(), k);
                std::exit(2);
            }
        };
        if (f == "--algo") { need(1); algo = argv[++i]; }
        else if (f == "--csv") { need(1); csv = argv[++i]; }
        else if (f == "--mode") { need(1); mode = argv[++i]; }
        else if (f == "--iters") { need(1); iters = std::atoi(argv[++i]); }
        else if (f == "--dt") { need(1); dt = std::strtod(argv[++i], nullptr); }
        else if (f == "--cutoff") { need(1); cutoff = std::strtod(argv[++i], nullptr); }
        else if (f == "--nu") { need(1); nu = std::strtod(argv[++i], nullptr); }
        else if (f == "--g") {
            need(3);
            for (int d = 0; d < 3; ++d) g[d] = std::strtod(argv[++i], nullptr);
        } else {
            std::fprintf(stderr, "ref_dump: unknown flag %s\n", f.c_str());
            return 2;
        }
    }
    if (csv.empty()) {
        std::fprintf(stderr, "ref_dump: --csv is required\n");
        return 2;
    }

    MPI_Init(&argc, &argv);
    MPI_Datatype particleType = Utility::Particle::GetMPIType();
    MPI_Type_commit(&particleType);

    std::vector<Utility::Particle> particles;
    Utility::getParticlesFromCSV(csv, particles);

    std::shared_ptr<Potential> potential = std::make_shared<AxilrodTeller>(nu);
    Eigen::Vector3d gForce(g[0], g[1], g[2]);
    std::shared_ptr<Simulation> sim;
    if (algo == "p3bca") {
        auto topo = std::make_shared<CartTopology>(std::vector<int>{1});
        auto decomp = std::make_shared<RegularGridDecomposition>();
        sim = std::make_shared<Simulation>(iters, std::make_shared<P3BCA>(cutoff), topo, potential, decomp,
                                           &particleType, particles, dt, gForce, "");
    } else {
        auto topo = std::make_shared<RingTopology>();
        auto decomp = std::make_shared<AtomDecomposition>();
        std::shared_ptr<Algorithm> alg;
        if (algo == "nata") alg = std::make_shared<NATA>();
        else alg = std::make_shared<AUTA>();
        sim = std::make_shared<Simulation>(iters, alg, topo, potential, decomp, &particleType, particles, dt, gForce,
                                           "");
    }
    sim->Init();

    auto t0 = std::chrono::steady_clock::now();
    std::vector<std::pair<uint64_t, uint64_t>> counts;
    if (mode == "forces") {
        auto r = sim->GetAlgorithm()->SimulationStep();
        counts.emplace_back(std::get<0>(r), std::get<1>(r));
    } else {
        sim->Start();
        for (int s = 0; s < iters; ++s)
            counts.emplace_back(sim->GetNumBufferInteractions(s), sim->GetNumParticleInteractions(s));
    }
    auto t1 = std::chrono::steady_clock::now();

    for (size_t s = 0; s < counts.size(); ++s)
        std::printf("step %zu buffer %llu triplets %llu\n", s, (unsigned long long)counts[s].first,
                    (unsigned long long)counts[s].second);
    std::vector<Utility::Particle> out = sim->GetDecomposition()->GetMyParticles();
    for (const Utility::Particle &p : out) {
        if (p.isDummy) continue;
        std::printf("particle %d %.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g\n", p.ID,
                    p.pX, p.pY, p.pZ, p.vX, p.vY, p.vZ, p.aX, p.aY, p.aZ, p.mass, p.fX, p.fY, p.fZ);
    }
    std::printf("time_ns %lld\n",
                (long long)std::chrono::duration_cast<std::chrono::nanoseconds>(t1 - t0).count());
    MPI_Type_free(&particleType);
    MPI_Finalize();
    return 0;
}
