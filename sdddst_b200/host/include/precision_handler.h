// Per-dislocation tolerance / error bookkeeping of the adaptive step
// (reference include/precision_handler.h:28-60).  The engine keeps its own
// device-side copy of this state; this host class serves API callers.
#ifndef SDDDST_B200_PRECISION_HANDLER_H
#define SDDDST_B200_PRECISION_HANDLER_H

#include <string>
#include <utility>
#include <vector>

namespace sdddstCore {

class PrecisionHandler
{
public:
    PrecisionHandler();
    ~PrecisionHandler();
    void setSize(unsigned int size);
    unsigned long getSize() const;
    void reset();
    void updateTolerance(const double &distanceSqr, const unsigned int &ID);
    void updateError(const double &error, const unsigned int &ID);
    double getNewStepSize(const double &oldStepSize) const;
    double getMinPrecisity() const;
    void setMinPrecisity(double value);
    double getMaxErrorRatioSqr() const;
    std::string __str__() const;
    std::string __repr__() const;

private:
    std::vector<std::pair<double, double>> toleranceAndError;
    double minPrecisity;
    double minPrecisitySqr;
    double maxErrorRatioSqr;
    unsigned int selectedID;
};

} // namespace sdddstCore

#endif
