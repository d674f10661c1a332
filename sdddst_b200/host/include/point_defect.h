// Fixed point defect of the host API (members as the reference's
// sdddstCore::PointDefect, include/point_defect.h:27-55).
#ifndef SDDDST_B200_POINT_DEFECT_H
#define SDDDST_B200_POINT_DEFECT_H

#include <string>

namespace sdddstCore {

struct PointDefect {
    double x;
    double y;
    bool operator==(PointDefect o) { return o.x == x && o.y == y; }
    std::string __repr__() const { return "x: " + std::to_string(x) + " y: " + std::to_string(y); }
    std::string __str__() const { return __repr__(); }
};

} // namespace sdddstCore

#endif
