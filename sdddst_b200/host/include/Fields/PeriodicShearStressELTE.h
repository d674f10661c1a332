// Tabulated periodic shear-stress field of the host API, the counterpart of
// the reference's sdddstCoreELTE::PeriodicShearStressELTE (loaded with
// loadStress(pwd, "xy", 1024) and loadStress(pwd, "xy_diff_x", 1024),
// python/src/periodic_shear_stress_ELTE_wrapper.cpp:40-46).  The reference
// ships neither the class's source nor its data file, so the tables are
// built from the analytic field: each holds the smooth remainder of the
// field after its image-free term on a 1024 x 1024 grid, and an evaluation
// adds that term in closed form to a bicubic interpolation of the remainder.
// The engine builds the same tables on the device (SDDDST_FIELD_TABULATED).
#ifndef SDDDST_B200_PERIODIC_SHEAR_STRESS_ELTE_H
#define SDDDST_B200_PERIODIC_SHEAR_STRESS_ELTE_H

#include <string>
#include <vector>

#include "Fields/Field.h"

namespace sdddstCoreELTE {

class PeriodicShearStressELTE : public sdddstCore::Field
{
public:
    PeriodicShearStressELTE();
    virtual ~PeriodicShearStressELTE();

    // Builds the table of `type` ("xy" or "xy_diff_x"); `size` must be 1024.
    // `path` names the directory of the reference's data file; its binary
    // format is not published, so no file is read and the table is computed.
    void loadStress(std::string path, std::string type, int size);

    virtual double xy(double dx, double dy);
    virtual double xy_diff_x(double dx, double dy);
    virtual int deviceKind() const;

private:
    std::vector<double> remXY, remDX;
};

} // namespace sdddstCoreELTE

#endif
