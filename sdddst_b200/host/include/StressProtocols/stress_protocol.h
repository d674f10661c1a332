// External stress protocols of the host API (reference
// include/StressProtocols/stress_protocol.h:31-82): the stage types and the
// zero-stress base class.  The engine evaluates the protocol of a
// simulation itself; deviceKind() names the device protocol (-1: none).
#ifndef SDDDST_B200_STRESS_PROTOCOL_H
#define SDDDST_B200_STRESS_PROTOCOL_H

#include "dislocation.h"

#include <string>
#include <vector>

namespace sdddstCore {

enum StressProtocolStepType { Original, EndOfBigStep, EndOfFirstSmallStep, EndOfSecondSmallStep };

class StressProtocol
{
public:
    StressProtocol();
    virtual ~StressProtocol();
    virtual void calculateStress(double simulationTime, const std::vector<Dislocation> &dislocations,
                                 StressProtocolStepType type);
    virtual double getStress(StressProtocolStepType type);
    virtual double getStressDerivative(double simulationTime);
    virtual bool getTriggerState();
    virtual std::string getType();
    virtual int deviceKind();
};

} // namespace sdddstCore

#endif
