// Spring-loaded external stress (reference
// include/StressProtocols/spring_protocol.h:28-43): k (rate t - strain),
// clamped at zero.
#ifndef SDDDST_B200_SPRING_PROTOCOL_H
#define SDDDST_B200_SPRING_PROTOCOL_H

#include "StressProtocols/fixed_rate_protocol.h"

namespace sdddstCore {

class SpringProtocol : public FixedRateProtocol
{
public:
    SpringProtocol();
    virtual ~SpringProtocol();
    using FixedRateProtocol::calculateStress;
    virtual void calculateStress(double simulationTime, const std::vector<Dislocation> &dislocations,
                                 StressProtocolStepType type, double strain);
    virtual std::string getType();
    virtual int deviceKind();
    double getSpringConstant() const;
    void setSpringConstant(double newSpringConstant);

protected:
    double springConstant;
};

} // namespace sdddstCore

#endif
