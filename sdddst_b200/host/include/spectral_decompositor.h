// The eigenvalue decomposition of a configuration's Hessian (the reference's
// sdddstEV::SpectralDecompositor, include/spectral_decompositor.h:27-66):
// same methods and meaning, the Hessian built and decomposed on the GPU
// (sdddst_ev_analyze).  The Field argument is taken over as in the reference;
// the device evaluates the analytic field (AnalyticField) only.
#ifndef SDDDST_B200_SPECTRAL_DECOMPOSITOR_H
#define SDDDST_B200_SPECTRAL_DECOMPOSITOR_H

#include "Fields/Field.h"
#include "dislocation.h"
#include "point_defect.h"

#include <memory>
#include <vector>

namespace sdddstEV {

struct Pair
{
    double eigen;
    unsigned long index;
};

class SpectralDecompositor
{
public:
    SpectralDecompositor(sdddstCore::Field *f);
    ~SpectralDecompositor();

    void decompose(std::vector<sdddstCore::Dislocation> &dislocations,
                   std::vector<sdddstCore::PointDefect> &pointDefects);

    double getEigenValue(unsigned int i);
    double getEigenVectorElement(int i, int j);

    unsigned long getDislocationCount() const;
    unsigned long getFpCount() const;

private:
    unsigned long dislocationCount;
    unsigned long fpCount;
    std::unique_ptr<sdddstCore::Field> field;
    void *ctx;
    std::vector<double> pdKey;
    std::vector<double> vectors; // eigenvector m at [m n ..]
    std::vector<Pair> eigenValues;
};

} // namespace sdddstEV

#endif
