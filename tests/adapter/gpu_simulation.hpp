// gpu_simulation.hpp: drop-in for Simulation::Init + Start + GetNumParticleInteractions
// (src/simulation/Simulation.cpp:3-96 of the reference) over the C ABI of include/tbmd.h.
#pragma once

#include <stdexcept>
#include <vector>

#include "tbmd.h"
#include "utility/structs.hpp"

class GpuSimulation {
public:
    GpuSimulation(int algorithm /* TBMD_NATA | TBMD_P3BCA | TBMD_AUTA, same numbering as AlgorithmType */,
                  std::vector<Utility::Particle> &particles, int iterations, double dt, double gx, double gy,
                  double gz, double cutoff, bool mixed = false)
        : particles_(particles), iterations_(iterations)
    {
        tbmd_config cfg;
        tbmd_config_init(&cfg);  // AUTA, FP64, nu = 1 (main.cpp:41,66,91), graphs on
        cfg.algorithm = algorithm;
        cfg.precision = mixed ? TBMD_MIXED : TBMD_FP64;
        cfg.cutoff = cutoff;
        cfg.dt = dt;
        cfg.g[0] = gx;
        cfg.g[1] = gy;
        cfg.g[2] = gz;
        check(tbmd_create(&cfg, &ctx_));
        const size_t n = particles.size();
        std::vector<int32_t> id(n);
        std::vector<double> f[10];
        for (auto &v : f) v.resize(n);
        for (size_t i = 0; i < n; ++i) {
            const Utility::Particle &p = particles[i];
            id[i] = p.ID;
            f[0][i] = p.pX; f[1][i] = p.pY; f[2][i] = p.pZ;
            f[3][i] = p.vX; f[4][i] = p.vY; f[5][i] = p.vZ;
            f[6][i] = p.aX; f[7][i] = p.aY; f[8][i] = p.aZ;
            f[9][i] = p.mass;
        }
        // for P3BCA this also fixes the periodic domain like RegularGridDecomposition::Init
        check(tbmd_set_particles(ctx_, (int64_t)n, id.data(), f[0].data(), f[1].data(), f[2].data(), f[3].data(),
                                 f[4].data(), f[5].data(), f[6].data(), f[7].data(), f[8].data(), f[9].data()));
    }
    ~GpuSimulation() { tbmd_destroy(ctx_); }

    // Simulation::Start: all iterations on the device, then the particles back into the vector
    void Start()
    {
        counts_.assign(iterations_, 0);
        check(tbmd_step(ctx_, iterations_, counts_.data()));
        const size_t n = particles_.size();
        std::vector<int32_t> id(n);
        std::vector<double> f[13];
        for (auto &v : f) v.resize(n);
        check(tbmd_get_particles(ctx_, id.data(), f[0].data(), f[1].data(), f[2].data(), f[3].data(), f[4].data(),
                                 f[5].data(), f[6].data(), f[7].data(), f[8].data(), f[9].data(), f[10].data(),
                                 f[11].data(), f[12].data()));
        for (size_t i = 0; i < n; ++i) {
            Utility::Particle &p = particles_[i];  // same order as given to tbmd_set_particles
            p.pX = f[0][i]; p.pY = f[1][i]; p.pZ = f[2][i];
            p.vX = f[3][i]; p.vY = f[4][i]; p.vZ = f[5][i];
            p.aX = f[6][i]; p.aY = f[7][i]; p.aZ = f[8][i];
            p.fX = f[10][i]; p.fY = f[11][i]; p.fZ = f[12][i];
        }
    }
    // Simulation::GetNumParticleInteractions (Simulation.cpp:93-96)
    uint64_t GetNumParticleInteractions(int step) const { return counts_.at(step); }

private:
    void check(tbmd_status s)
    {
        // the reference prints and exit(1)s on bad input; an exception lets the caller choose
        if (s != TBMD_OK) throw std::runtime_error(ctx_ ? tbmd_last_error(ctx_) : tbmd_status_string(s));
    }
    tbmd_ctx *ctx_ = nullptr;
    std::vector<Utility::Particle> &particles_;
    int iterations_;
    std::vector<uint64_t> counts_;
};
