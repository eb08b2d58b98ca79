// Rank-layout driver around the reference's own set-up code (test infrastructure only).
//
// Run under the stub MPI's layout mode (TBMD_STUB_WORLD_SIZE=P, TBMD_STUB_RANK=r), it wires the
// Simulation of one algorithm exactly as the reference's main does (src/main.cpp:32-105, 546-551:
// RingTopology + AtomDecomposition for NATA / AUTA, CartTopology over
// Utility::getDecomposition(P, table) + RegularGridDecomposition for P3BCA) and calls
// Simulation::Init (Simulation.cpp:12-19), which runs the topology's, the decomposition's and the
// algorithm's set-up for rank r.  Where the reference stops (P3BCA.cpp:53-70,
// CartTopology.cpp:55-57) it stops the same way: its message on stderr and exit status 1.
// Otherwise it prints one JSON line with what set-up decided.
//
//   ref_layout --tables            both process-grid tables for P = 1..1030, one JSON line
//   ref_layout --algo nata|auta|p3bca --csv FILE [--cutoff C] [--decomp optimal|naive]
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
#include "utility/decompositions.hpp"
#include "utility/utility.hpp"

static void print_grid(const std::vector<int> &d)
{
    std::printf("[");
    for (size_t i = 0; i < d.size(); ++i) std::printf("%s%d", i ? ", " : "", d[i]);
    std::printf("]");
}

int main(int argc, char **argv)
{
    std::string algo = "p3bca", csv, decomp = "naive";
    double cutoff = 0.0;
    bool tables = false;
    for (int i = 1; i < argc; ++i) {
        std::string f = argv[i];
        if (f == "--tables") tables = true;
        else if (f == "--algo" && i + 1 < argc) algo = argv[++i];
        else if (f == "--csv" && i + 1 < argc) csv = argv[++i];
        else if (f == "--cutoff" && i + 1 < argc) cutoff = std::strtod(argv[++i], nullptr);
        else if (f == "--decomp" && i + 1 < argc) decomp = argv[++i];
        else {
            std::fprintf(stderr, "ref_layout: bad argument %s\n", f.c_str());
            return 2;
        }
    }
    if (tables) {
        std::printf("{\"optimal\": {");
        for (int P = 1; P <= 1030; ++P) {
            std::printf("%s\"%d\": ", P > 1 ? ", " : "", P);
            print_grid(Utility::getDecomposition(P, decompositions));
        }
        std::printf("}, \"naive\": {");
        for (int P = 1; P <= 1030; ++P) {
            std::printf("%s\"%d\": ", P > 1 ? ", " : "", P);
            print_grid(Utility::getDecomposition(P, decompositionsNaive));
        }
        std::printf("}}\n");
        return 0;
    }
    if (csv.empty()) {
        std::fprintf(stderr, "ref_layout: --csv is required\n");
        return 2;
    }

    MPI_Init(&argc, &argv);
    int worldSize = 1;
    MPI_Comm_size(MPI_COMM_WORLD, &worldSize);
    MPI_Datatype particleType = Utility::Particle::GetMPIType();
    MPI_Type_commit(&particleType);
    std::vector<Utility::Particle> particles;
    Utility::getParticlesFromCSV(csv, particles);

    std::shared_ptr<Potential> potential = std::make_shared<AxilrodTeller>(1.0);
    Eigen::Vector3d gForce(0.0, 0.0, 0.0);
    std::shared_ptr<Simulation> sim;
    std::shared_ptr<CartTopology> cart;
    std::shared_ptr<P3BCA> p3bca;
    std::vector<int> grid;
    if (algo == "p3bca") {
        grid = Utility::getDecomposition(worldSize, decomp == "optimal" ? decompositions : decompositionsNaive);
        cart = std::make_shared<CartTopology>(grid);
        p3bca = std::make_shared<P3BCA>(cutoff);
        sim = std::make_shared<Simulation>(1, p3bca, cart, potential, std::make_shared<RegularGridDecomposition>(),
                                           &particleType, particles, 0.001, gForce, "");
    } else {
        std::shared_ptr<Algorithm> alg;
        if (algo == "nata") alg = std::make_shared<NATA>();
        else alg = std::make_shared<AUTA>();
        sim = std::make_shared<Simulation>(1, alg, std::make_shared<RingTopology>(),
                                           potential, std::make_shared<AtomDecomposition>(), &particleType, particles,
                                           0.001, gForce, "");
    }
    sim->Init();

    const std::vector<Utility::Particle> mine = sim->GetDecomposition()->GetMyParticles();
    long long dummies = 0;
    for (const Utility::Particle &p : mine) dummies += p.isDummy ? 1 : 0;
    std::printf("{\"world_size\": %d, \"my_particles\": %zu, \"my_dummies\": %lld", worldSize, mine.size(), dummies);
    if (p3bca) {
        const std::array<int, 3> nCb = p3bca->GetNumCutoffBoxes();
        const std::array<int, 3> dims = cart->GetDims();
        std::printf(", \"grid\": ");
        print_grid(grid);
        std::printf(", \"dims\": [%d, %d, %d], \"cutoff_boxes\": [%d, %d, %d]", dims[0], dims[1], dims[2], nCb[0],
                    nCb[1], nCb[2]);
    }
    std::printf("}\n");
    MPI_Type_free(&particleType);
    MPI_Finalize();
    return 0;
}
