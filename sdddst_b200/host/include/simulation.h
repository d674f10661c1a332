// The implicit step driver of the host API (the reference's
// sdddstCore::Simulation, include/simulation.h:38-86), running on a B200
// through the engine's C ABI (include/sdddst_b200.h).  Same methods and
// meaning; the engine context is created from SimulationData on
// construction and the SimulationData vectors are refreshed from the device
// after every step.  Engine failures throw sdddstCore::EngineError (the
// reference ignores the UMFPACK status instead).
#ifndef SDDDST_B200_SIMULATION_H
#define SDDDST_B200_SIMULATION_H

#include "StressProtocols/stress_protocol.h"
#include "dislocation.h"
#include "precision_handler.h"
#include "simulation_data.h"

#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace sdddstCore {

class EngineError : public std::runtime_error
{
public:
    EngineError(int code, const std::string &msg) : std::runtime_error(msg), code(code) {}
    int code;
};

class Simulation
{
public:
    Simulation(std::shared_ptr<SimulationData> _sD);
    ~Simulation();

    void integrate(const double &stepsize, std::vector<Dislocation> &newDislocation,
                   const std::vector<Dislocation> &old, bool useSpeed2, bool calculateInitSpeed,
                   StressProtocolStepType origin, StressProtocolStepType end);
    void calculateSpeeds(const std::vector<Dislocation> &dis, std::vector<double> &res, bool ignorePHUpdate = false);
    void calculateG(const double &stepsize, std::vector<Dislocation> &newDislocation,
                    const std::vector<Dislocation> &old, bool useSpeed2, bool calculateInitSpeed,
                    bool useInitSpeedForFirstStep, StressProtocolStepType origin, StressProtocolStepType end);
    void calculateJacobian(const double &stepsize, const std::vector<Dislocation> &data);
    void calculateXError();
    void calculateSparseFormForJacobian();
    void solveEQSys();
    double calculateOrderParameter(const std::vector<double> &speeds);
    double getElement(int j, int si, int ei);
    double getSimTime();
    void run();
    bool step();
    void stepStageI();
    void stepStageII();
    void stepStageIII();
    const std::vector<Dislocation> &getStoredDislocationData();

    // engine options used when the context is created (pair-sum and solver
    // arithmetic, see sdddst_params); call before the first step.
    void setEngineOptions(int pairsum, int solver, double solverTol);
    // per-dislocation tolerances of the last step (PrecisionHandler state)
    std::vector<double> lastTolerances();
    double lastMaxErrorRatioSqr();

private:
    void ensureContext();
    void pushState();
    void pullState();
    void afterAcceptedStep(double wallStart);
    void check(int rc);

    bool succesfulStep;
    double lastWriteTimeFinished;
    bool initSpeedCalculationIsNeeded;
    bool firstStepRequest;
    double energy;
    double energyAccum;
    double vsquare;

    std::shared_ptr<SimulationData> sD;
    std::unique_ptr<PrecisionHandler> pH;
    void *ctx;
    int optPairsum, optSolver;
    double optSolverTol;
    std::vector<Dislocation> pushed; // configuration the device holds
    double pushedStep, pushedTime;
    bool stagedThisStep;
};

} // namespace sdddstCore

#endif
