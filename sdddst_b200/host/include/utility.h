// Host helpers of the reference's include/utility.h:29-100 (minimum image,
// periodic distance kernels X, X2, E and their x-derivatives, wall/cpu
// clocks, strain increment), same names and meaning.
#ifndef SDDDST_B200_UTILITY_H
#define SDDDST_B200_UTILITY_H

#include <cmath>
#include <ctime>
#include <sys/time.h>
#include <vector>

#include "dislocation.h"

// minimum image into [-0.5, 0.5)
inline void normalize(double &n)
{
    if (!std::isfinite(n)) return;
    if (std::fabs(n) >= 8.0) n -= std::floor(n);
    while (n < -0.5) n += 1.0;
    while (n >= 0.5) n -= 1.0;
}

inline double X(const double &x) { return std::sin(2.0 * M_PI * x) * 0.5 / M_PI; }
inline double X2(const double &x) { return (1.0 - std::cos(2.0 * M_PI * x)) * 0.5 / M_PI / M_PI; }
inline double E(const double &x, const double &y, const double &K) { return std::exp(-K * (X2(x) + X2(y))); }
inline double X_dx(const double &x) { return std::cos(2.0 * M_PI * x); }
inline double X2_dx(const double &x) { return std::sin(2.0 * M_PI * x) / M_PI; }
inline double E_dx(const double &x, const double &y, const double &K) { return -E(x, y, K) * K * X2_dx(x); }

inline double get_wall_time()
{
    struct timeval t;
    if (gettimeofday(&t, nullptr)) return 0;
    return (double)t.tv_sec + (double)t.tv_usec * 1e-6;
}

inline double get_cpu_time() { return (double)std::clock() / CLOCKS_PER_SEC; }

// sum_i b_i (x_new,i - x_old,i)
inline double calculateStrainIncrement(const std::vector<sdddstCore::Dislocation> &old,
                                       const std::vector<sdddstCore::Dislocation> &newD)
{
    double s = 0;
    for (size_t i = 0; i < old.size(); ++i) s += newD[i].b * (newD[i].x - old[i].x);
    return s;
}

#endif
