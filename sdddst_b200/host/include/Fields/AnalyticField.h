// Analytic periodic stress field (reference include/Fields/AnalyticField.h):
// tau_xy of an edge dislocation summed over y-periodic image columns at
// dx + k, |k| <= ANALYTIC_FIELD_N, with the reference's end weighting.  The
// host evaluations here serve API callers; the simulation itself uses the
// device kernels (SDDDST_FIELD_ANALYTIC).
#ifndef SDDDST_B200_ANALYTIC_FIELD_H
#define SDDDST_B200_ANALYTIC_FIELD_H

#include "Fields/Field.h"
#include "constants.h"

#include <cmath>

namespace sdddstCore {

class AnalyticField : public Field
{
public:
    AnalyticField();
    virtual ~AnalyticField();

    virtual double xy(double dx, double dy);
    virtual double xy_diff_x(double dx, double dy);
    // second x-derivative by Richardson extrapolation of xy_diff_x
    virtual double xy_diff_x2(double dx, double dy);

    virtual int deviceKind() const;
};

} // namespace sdddstCore

#endif
