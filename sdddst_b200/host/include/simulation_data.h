// State and parameters of one simulated system (the reference's
// sdddstCore::SimulationData, include/simulation_data.h:39-280): same public
// members, so code written against the reference's SimulationData compiles
// unchanged.  The CSC arrays Ap/Ai/Ax hold the Jacobian of the last
// Simulation::calculateJacobian call (the reference's UMFPACK layout); the
// UMFPACK handles are kept for source compatibility and stay null.
#ifndef SDDDST_B200_SIMULATION_DATA_H
#define SDDDST_B200_SIMULATION_DATA_H

#include "Fields/Field.h"
#include "StressProtocols/stress_protocol.h"
#include "dislocation.h"
#include "point_defect.h"

#include <fstream>
#include <memory>
#include <string>
#include <vector>

namespace sdddstCore {

class SimulationData
{
public:
    SimulationData(const std::string &dislocationDataFilePath, const std::string &pointDefectDataFilePath);
    SimulationData();
    ~SimulationData();

    void readDislocationDataFromFile(const std::string &dislocationDataFilePath);
    void writeDislocationDataToFile(const std::string &dislocationDataFilePath);
    void readPointDefectDataFromFile(const std::string &pointDefectDataFilePath);
    void writePointDefectDataToFile(const std::string &pointDefectDataFilePath);
    void initSimulationVariables();
    void updateCutOff();

    std::vector<Dislocation> dislocations;
    std::vector<PointDefect> points;
    std::vector<double> g;
    std::vector<double> initSpeed;
    std::vector<double> initSpeed2;
    std::vector<double> speed;
    std::vector<double> speed2;
    std::vector<double> dVec;
    double cutOffMultiplier;
    double cutOff;
    double cutOffSqr;
    double onePerCutOffSqr;
    double prec;
    unsigned int pc;
    unsigned int dc;
    unsigned int ic;
    double timeLimit;
    double stepSize;
    double simTime;
    double KASQR;
    double A;
    std::vector<Dislocation> bigStep;
    std::vector<Dislocation> firstSmall;
    std::vector<Dislocation> secondSmall;
    std::unique_ptr<Field> tau;
    int *Ap;
    int *Ai;
    double *Ax;
    double *x;
    double *null;
    void *Symbolic, *Numeric;
    std::vector<int> indexes;
    size_t succesfulSteps;
    size_t failedSteps;
    double totalAccumulatedStrainIncrease;
    bool isStrainIncreaseLimit;
    double totalAccumulatedStrainIncreaseLimit;
    bool isMaxStepSizeLimit;
    double maxStepSizeLimit;
    bool isTimeLimit;
    bool isStepCountLimit;
    unsigned int stepCountLimit;
    bool isSpeedLimit;
    bool finish;
    double speedLimit;
    double stressLimit;
    bool isStressLimit;
    bool calculateStrainDuringSimulation;
    bool orderParameterCalculationIsOn;
    std::ofstream standardOutputLog;
    std::string endDislocationConfigurationPath;
    std::unique_ptr<StressProtocol> externalStressProtocol;
    bool countAvalanches;
    double avalancheSpeedThreshold;
    unsigned int avalancheTriggerLimit;
    unsigned int avalancheCount;
    bool inAvalanche;
    bool isSaveSubConfigs;
    std::string subConfigPath;
    unsigned int subConfigDelay;
    unsigned int subConfigDelayDuringAvalanche;
    unsigned int subconfigDistanceCounter;
    StressProtocolStepType currentStressStateType;
    double speedThresholdForCutoffChange;
    bool isSpeedThresholdForCutoffChange;
    unsigned currentStorageSize;
    double sumAvgSpeed;
    std::string eVAnalResultFile;
    unsigned int remainingFinalSteps;
    bool inFinal;
    bool calculateDerivativeEVAnal;
    int numberOfEigenVecToWrite;
    int writeCorrelMatrices;

    // number of stored entries of Ap/Ai/Ax (nnz after the last assembly)
    long jacobianNonZeros;

private:
    void resizeForDislocationCount();
    void releaseJacobian();
};

} // namespace sdddstCore

#endif
