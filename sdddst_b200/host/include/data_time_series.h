// The list of saved configurations the eigenvalue analysis walks through
// (the reference's DataTimeSeries, include/data_time_series.h,
// src/data_time_series.cpp:1-42): a text file of "time path" pairs, each
// read with the point-defect file into SimulationData by next().
#ifndef SDDDST_B200_DATA_TIME_SERIES_H
#define SDDDST_B200_DATA_TIME_SERIES_H

#include "simulation_data.h"

#include <list>
#include <memory>
#include <string>

class DataTimeSeries
{
public:
    DataTimeSeries(std::string dconfList, std::string fconf = "");

    bool next(std::shared_ptr<sdddstCore::SimulationData> sD);

private:
    std::list<std::pair<double, std::string>> dconfs;
    std::string fconfPath;
};

#endif
