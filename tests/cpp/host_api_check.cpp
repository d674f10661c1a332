// Drives the reference-named C++ API (sdddstCore::Simulation and friends)
// on a configuration file and prints the results of its fine-grained
// operations, for tests/test_host_api.py to compare with the oracle:
//   speeds <N values>            Simulation::calculateSpeeds
//   csc <N+1 Ap> <nnz Ai> <nnz Ax> <N dVec>   Simulation::calculateJacobian
//   integrate <N x>              Simulation::integrate (big step, h)
// usage: host_api_check <dconf> <cutoff multiplier> <prec> <h>
#include "Fields/AnalyticField.h"
#include "simulation.h"

#include <cstdio>
#include <cstdlib>
#include <memory>

using namespace sdddstCore;

int main(int argc, char **argv)
{
    if (argc < 5) return 2;
    auto sd = std::make_shared<SimulationData>(argv[1], "");
    sd->cutOffMultiplier = std::atof(argv[2]);
    sd->updateCutOff();
    sd->prec = std::atof(argv[3]);
    sd->stepSize = std::atof(argv[4]);
    sd->tau.reset(new AnalyticField());
    sd->externalStressProtocol.reset(new StressProtocol());
    Simulation sim(sd);
    try {
        std::vector<double> v;
        sim.calculateSpeeds(sd->dislocations, v);
        std::printf("speeds");
        for (double a : v) std::printf(" %.17g", a);
        std::printf("\n");
        sim.calculateJacobian(sd->stepSize, sd->dislocations);
        const int n = (int)sd->dc;
        const long nnz = sd->Ap[n];
        std::printf("csc %d %ld", n, nnz);
        for (int j = 0; j <= n; ++j) std::printf(" %d", sd->Ap[j]);
        for (long q = 0; q < nnz; ++q) std::printf(" %d", sd->Ai[q]);
        for (long q = 0; q < nnz; ++q) std::printf(" %.17g", sd->Ax[q]);
        for (int j = 0; j < n; ++j) std::printf(" %.17g", sd->dVec[j]);
        std::printf("\n");
        // stage I of a fresh step: initial speeds, then integrate(h, bigStep, dislocations)
        sim.calculateSpeeds(sd->dislocations, sd->initSpeed);
        sd->bigStep = sd->dislocations;
        sim.integrate(sd->stepSize, sd->bigStep, sd->dislocations, false, false, Original, EndOfBigStep);
        std::printf("integrate");
        for (auto &d : sd->bigStep) std::printf(" %.17g", d.x);
        std::printf("\n");
    } catch (const EngineError &e) {
        std::fprintf(stderr, "engine error %d: %s\n", e.code, e.what());
        return 1;
    }
    return 0;
}
