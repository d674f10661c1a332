// Edge dislocation record of the host API (same layout and members as the
// reference's sdddstCore::Dislocation, include/dislocation.h:27-55).
#ifndef SDDDST_B200_DISLOCATION_H
#define SDDDST_B200_DISLOCATION_H

#include <string>

namespace sdddstCore {

struct Dislocation {
    double x;
    double y;
    double b;
    bool operator==(Dislocation o) { return o.x == x && o.y == y && o.b == b; }
    std::string __str__() const
    {
        return "x: " + std::to_string(x) + " y: " + std::to_string(y) + " b: " + std::to_string(b);
    }
    std::string __repr__() const { return __str__(); }
};

} // namespace sdddstCore

#endif
