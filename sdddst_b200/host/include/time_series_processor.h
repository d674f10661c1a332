// The eigenvalue analysis run (the reference's sdddstEV::TimeSeriesProcessor,
// include/time_series_processor.h, src/time_series_processor.cpp:21-204): for
// every configuration of the series, the eigenvalues, participation numbers,
// 1/Gael, velocities, x coordinates, Burgers sums, the first eigenvectors and
// optionally the eigenvalue derivatives -- or, with writeCorrelMatrices, the
// correlation matrices -- as text lines into a gzip file, in the reference's
// format.  Everything per configuration is computed by one device call
// (sdddst_ev_analyze).
#ifndef SDDDST_B200_TIME_SERIES_PROCESSOR_H
#define SDDDST_B200_TIME_SERIES_PROCESSOR_H

#include "StressProtocols/stress_protocol.h"
#include "data_time_series.h"
#include "simulation.h"
#include "simulation_data.h"

#include <memory>

namespace sdddstEV {

class TimeSeriesProcessor
{
public:
    TimeSeriesProcessor(std::shared_ptr<sdddstCore::SimulationData> sD, std::shared_ptr<DataTimeSeries> dateTimeSeries,
                        sdddstCore::StressProtocol *stressProtocol);
    ~TimeSeriesProcessor();

    void run();

    std::shared_ptr<sdddstCore::Simulation> sim;

private:
    std::shared_ptr<sdddstCore::SimulationData> sD;
    std::shared_ptr<DataTimeSeries> dTS;
    void *ctx;
    int ctxN, ctxP;
};

} // namespace sdddstEV

#endif
