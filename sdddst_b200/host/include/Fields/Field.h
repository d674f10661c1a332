// Field plug-in of the host API (reference include/Fields/Field.h:28-37):
// virtual per-pair stress evaluations.  The engine cannot call a host
// virtual per pair, so each field also names the device kernel that
// implements it (deviceKind(): an SDDDST_FIELD_* value, or -1 when there is
// none; Simulation refuses such a field rather than running on the CPU).
#ifndef SDDDST_B200_FIELD_H
#define SDDDST_B200_FIELD_H

namespace sdddstCore {

class Field
{
public:
    Field();
    virtual ~Field();

    virtual double xy(double dx, double dy);
    virtual double xy_diff_x(double dx, double dy);
    virtual double xy_diff_x2(double dx, double dy);

    virtual int deviceKind() const;
};

} // namespace sdddstCore

#endif
