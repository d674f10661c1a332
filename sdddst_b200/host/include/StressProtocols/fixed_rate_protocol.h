// Linearly increasing external stress (reference
// include/StressProtocols/fixed_rate_protocol.h:27-45), and the constant
// stress used for loaded runs (no counterpart in the reference, whose
// protocols are zero, fixed rate and spring).
#ifndef SDDDST_B200_FIXED_RATE_PROTOCOL_H
#define SDDDST_B200_FIXED_RATE_PROTOCOL_H

#include "StressProtocols/stress_protocol.h"

namespace sdddstCore {

class FixedRateProtocol : public StressProtocol
{
public:
    FixedRateProtocol();
    virtual ~FixedRateProtocol();
    virtual void calculateStress(double simulationTime, const std::vector<Dislocation> &dislocations,
                                 StressProtocolStepType type);
    virtual double getStress(StressProtocolStepType type);
    virtual double getStressDerivative(double simulationTime);
    virtual std::string getType();
    virtual int deviceKind();
    double getRate() const;
    void setRate(double value);

protected:
    double rate;
    double stressValues[4];
};

class ConstantStressProtocol : public StressProtocol
{
public:
    explicit ConstantStressProtocol(double value = 0.0);
    virtual double getStress(StressProtocolStepType type);
    virtual std::string getType();
    virtual int deviceKind();
    double getValue() const;
    void setValue(double v);

protected:
    double value;
};

} // namespace sdddstCore

#endif
