// sdddst -- command-line drop-in for the reference's `sdddst` simulation mode
// (src/main.cpp:22-45, src/project_parser.cpp:33-298), on the GPU engine.
//
// The reference parses its options with boost::program_options; Boost is not
// available here, so the same option names, argument types, defaults and
// checks are parsed by hand: `--name value` and `--name=value`, unambiguous
// prefixes of a long name (program_options' default guessing), `-c` for
// --hide-copyright.  Option semantics follow ProjectParser::processInput
// (project_parser.cpp:137-298) field by field; the run is Simulation::run and
// the log is the reference's 12-column log (simulation.cpp:463-617), written
// by the host API.  The eigenvalue analysis mode (--ev-analyzation) follows
// the EV branch of processInput (:299-318) and main (src/main.cpp:36-41) and
// runs TimeSeriesProcessor on the GPU.
#include "Fields/AnalyticField.h"
#include "StressProtocols/fixed_rate_protocol.h"
#include "StressProtocols/spring_protocol.h"
#include "StressProtocols/stress_protocol.h"
#include "data_time_series.h"
#include "simulation.h"
#include "simulation_data.h"
#include "time_series_processor.h"

#include <cmath>
#include <cstdio>
#include <exception>
#include <cstdlib>
#include <iostream>
#include <map>
#include <memory>
#include <string>
#include <vector>

using namespace sdddstCore;

namespace {

enum class Arg { None, Double, Unsigned, Int, String };

struct Opt {
    const char *name;
    Arg arg;
    const char *deflt; // default value (program_options default_value), or nullptr
    const char *help;
};

// The option table of project_parser.cpp:39-99 (simulation and EV modes).
const Opt kOpts[] = {
    {"simulation", Arg::None, nullptr, "run a simulation (default)"},
    {"ev-analyzation", Arg::None, nullptr, "run eigen value analysation"},
    {"dislocation-configuration", Arg::String, nullptr, "plain text file path containing dislocation data in {x y b} triplets"},
    {"result-dislocation-configuration", Arg::String, nullptr, "path where the result configuration will be stored at the end of the simulation"},
    {"point-defect-configuration", Arg::String, nullptr, "plain text file path containing point defect data in {x y} pairs"},
    {"logfile-path", Arg::String, nullptr, "path for the plain text log file (it will be overwritten if it already exists)"},
    {"time-limit", Arg::Double, nullptr, "in simulation time limit, if reached the simulation stops"},
    {"speed-limit", Arg::Double, nullptr, "in simulation units, if |v| falls below, the simulation stops"},
    {"step-count-limit", Arg::Unsigned, nullptr, "the simulation will stop after successful N steps"},
    {"strain-increase-limit", Arg::Double, nullptr, "the simulation will stop after arg total strain increase is reached"},
    {"stress-limit", Arg::Double, nullptr, "the simulation will stop after arg external stress is reached"},
    {"avalanche-detection-limit", Arg::Unsigned, nullptr, "the simulation will stop after the threshold was reached with the given number of events from above"},
    {"avalanche-speed-threshold", Arg::Double, "1e-3", "speed threshold for counting avalanches"},
    {"initial-stepsize", Arg::Double, "1e-6", "first tried step size for the simulation"},
    {"cutoff-multiplier", Arg::Double, "1e20", "multiplier of the 1/sqrt(N) cutoff parameter"},
    {"max-stepsize", Arg::Double, nullptr, "the stepsize can not overleap this value"},
    {"calculate-strain", Arg::None, nullptr, "turns on strain calculation for the simulation"},
    {"calculate-order-parameter", Arg::None, nullptr, "turns on order parameter calculation during the simulation"},
    {"position-precision", Arg::Double, "1e-5", "minimum precision for the positions for the adaptive step size protocol"},
    {"save-sub-configurations", Arg::String, nullptr, "saves the current configuration after every N successful step to the given destination"},
    {"sub-configuration-delay", Arg::Unsigned, "5", "number of successful steps between the sub configurations written out"},
    {"sub-configuration-delay-during-avalanche", Arg::Unsigned, "1", "number of successful steps between the sub configurations written out during avalanche if avalanche detection is on"},
    {"change-cutoff-to-inf-under-threshold", Arg::Double, nullptr, "if the avg speed decreases once under this threshold during the simulation the applied cutoff multiplier will be 1e20"},
    {"post-relax", Arg::Unsigned, "0", "Number of extra steps after finish condition is reached"},
    {"periodic-stress-field-analytic", Arg::None, nullptr, "analytic periodic stress field (default)"},
    {"no-external-stress", Arg::None, nullptr, "no external stress during the simulation (default)"},
    {"fixed-rate-external-stress", Arg::Double, nullptr, "external stress is linear with time, rate should be specified as an arg"},
    {"spring-constant", Arg::Double, nullptr, "simple model of an experiment where a spring is used, the arg should be the spring constant (it is valid only with the previous option together)"},
    {"file-list", Arg::String, nullptr, "file list with timestamps (EV analysis)"},
    {"pd-configuration", Arg::String, nullptr, "file path to the point defect config file (EV analysis)"},
    {"result-ev-file", Arg::String, nullptr, "file path where to save result (EV analysis)"},
    {"calculate-ev-deriv", Arg::None, nullptr, "EV derivative calculation (EV analysis)"},
    {"eigenvector-to-write", Arg::Int, "10", "number of eigenvectors to write into file (EV analysis)"},
    {"write-correlation-matrices", Arg::Int, nullptr, "write correlation matrices (EV analysis)"},
    {"help", Arg::None, nullptr, "show this help"},
    {"hide-copyright", Arg::None, nullptr, "hides the copyright notice from the standard output (short: -c)"},
};

struct Values {
    std::map<std::string, std::string> given; // options on the command line (value or "")
    std::map<std::string, int> count;
    bool has(const std::string &k) const { return count.count(k) && count.at(k) > 0; }
    std::string raw(const std::string &k) const
    {
        auto it = given.find(k);
        if (it != given.end()) return it->second;
        for (const Opt &o : kOpts)
            if (k == o.name && o.deflt) return o.deflt;
        return "";
    }
};

[[noreturn]] void die(const std::string &msg, int code)
{
    std::cerr << msg << std::endl;
    std::exit(code);
}

const Opt *find_opt(const std::string &name)
{
    for (const Opt &o : kOpts)
        if (name == o.name) return &o;
    // unambiguous prefix (program_options' guessing)
    const Opt *hit = nullptr;
    int hits = 0;
    for (const Opt &o : kOpts)
        if (std::string(o.name).compare(0, name.size(), name) == 0) {
            hit = &o;
            ++hits;
        }
    if (hits > 1) die("option '--" + name + "' is ambiguous", -1);
    return hit;
}

double as_double(const Values &v, const std::string &k)
{
    const std::string s = v.raw(k);
    char *end = nullptr;
    const double d = std::strtod(s.c_str(), &end);
    if (s.empty() || *end != '\0') die("the argument ('" + s + "') for option '--" + k + "' is invalid", -1);
    return d;
}

unsigned as_unsigned(const Values &v, const std::string &k)
{
    const std::string s = v.raw(k);
    char *end = nullptr;
    const long long d = std::strtoll(s.c_str(), &end, 10);
    if (s.empty() || *end != '\0' || d < 0 || d > 4294967295LL)
        die("the argument ('" + s + "') for option '--" + k + "' is invalid", -1);
    return (unsigned)d;
}

Values parse(int argc, char **argv)
{
    Values v;
    for (int a = 1; a < argc; ++a) {
        std::string tok = argv[a];
        std::string name, val;
        bool has_val = false;
        if (tok == "-c") {
            name = "hide-copyright";
        } else if (tok.size() > 2 && tok.compare(0, 2, "--") == 0) {
            name = tok.substr(2);
            const size_t eq = name.find('=');
            if (eq != std::string::npos) {
                val = name.substr(eq + 1);
                name = name.substr(0, eq);
                has_val = true;
            }
        } else {
            die("unrecognised option '" + tok + "'", -1);
        }
        const Opt *o = find_opt(name);
        if (!o) die("unrecognised option '--" + name + "'", -1);
        if (o->arg == Arg::None) {
            if (has_val) die("option '--" + std::string(o->name) + "' does not take any arguments", -1);
        } else if (!has_val) {
            if (a + 1 >= argc) die("the required argument for option '--" + std::string(o->name) + "' is missing", -1);
            val = argv[++a];
        }
        if (o->arg != Arg::None && v.count[o->name] > 0 && o->arg != Arg::String)
            die("option '--" + std::string(o->name) + "' cannot be specified more than once", -1);
        v.count[o->name]++;
        v.given[o->name] = val;
        // typed values are converted when stored, as program_options does
        if (o->arg == Arg::Double) (void)as_double(v, o->name);
        if (o->arg == Arg::Unsigned) (void)as_unsigned(v, o->name);
        if (o->arg == Arg::Int) {
            char *end = nullptr;
            (void)std::strtol(val.c_str(), &end, 10);
            if (val.empty() || *end != '\0')
                die("the argument ('" + val + "') for option '--" + std::string(o->name) + "' is invalid", -1);
        }
    }
    return v;
}

void print_help()
{
    std::cout << "sdddst (B200 engine) options:\n";
    for (const Opt &o : kOpts) {
        std::cout << "  --" << o.name;
        if (o.arg != Arg::None) std::cout << " arg";
        if (o.deflt) std::cout << " (=" << o.deflt << ")";
        std::cout << "\n      " << o.help << "\n";
    }
}

// ProjectParser::processInput (project_parser.cpp:137-298), simulation mode
std::shared_ptr<SimulationData> simulation_data(const Values &vm)
{
    if (!vm.has("dislocation-configuration")) die("dislocation-configuration is missing!", -1);
    if (!vm.has("result-dislocation-configuration")) die("result-dislocation-configuration is missing!", -1);
    std::shared_ptr<SimulationData> sD;
    if (vm.has("point-defect-configuration")) {
        if (vm.count.at("point-defect-configuration") > 1) die("Multiple definition of point-defect-configuration", 2);
        sD = std::make_shared<SimulationData>(vm.raw("dislocation-configuration"), vm.raw("point-defect-configuration"));
    } else {
        sD = std::make_shared<SimulationData>(vm.raw("dislocation-configuration"), "");
    }
    if (vm.has("time-limit")) {
        sD->isTimeLimit = true;
        sD->timeLimit = as_double(vm, "time-limit");
    }
    sD->stepSize = as_double(vm, "initial-stepsize"); // always present (default 1e-6)
    if (vm.has("stress-limit")) {
        sD->stressLimit = as_double(vm, "stress-limit");
        sD->isStressLimit = true;
    }
    sD->prec = as_double(vm, "position-precision"); // default 1e-5
    sD->cutOffMultiplier = as_double(vm, "cutoff-multiplier"); // default 1e20
    sD->updateCutOff();
    if (vm.has("strain-increase-limit")) {
        sD->isStrainIncreaseLimit = true;
        sD->totalAccumulatedStrainIncreaseLimit = as_double(vm, "strain-increase-limit");
    }
    if (vm.has("max-stepsize")) {
        sD->maxStepSizeLimit = as_double(vm, "max-stepsize");
        sD->isMaxStepSizeLimit = true;
    }
    if (vm.has("point-defect-configuration")) {
        sD->A *= 1. / std::sqrt((double)sD->dc);
        sD->KASQR *= double(sD->dc);
    }
    if (vm.has("calculate-strain")) sD->calculateStrainDuringSimulation = true;
    if (vm.has("calculate-order-parameter")) sD->orderParameterCalculationIsOn = true;
    if (vm.has("logfile-path")) sD->standardOutputLog = std::ofstream(vm.raw("logfile-path"));
    if (vm.has("step-count-limit")) {
        sD->isStepCountLimit = true;
        sD->stepCountLimit = as_unsigned(vm, "step-count-limit");
    }
    if (vm.has("avalanche-detection-limit")) {
        sD->countAvalanches = true;
        sD->avalancheTriggerLimit = as_unsigned(vm, "avalanche-detection-limit");
        sD->avalancheSpeedThreshold = as_double(vm, "avalanche-speed-threshold");
    }
    if (vm.has("save-sub-configurations")) {
        sD->isSaveSubConfigs = true;
        sD->subConfigPath = vm.raw("save-sub-configurations");
        sD->subConfigDelay = as_unsigned(vm, "sub-configuration-delay");
        sD->subConfigDelayDuringAvalanche = as_unsigned(vm, "sub-configuration-delay-during-avalanche");
    }
    if (vm.has("speed-limit")) {
        sD->isSpeedLimit = true;
        sD->speedLimit = as_double(vm, "speed-limit");
    }
    sD->remainingFinalSteps = as_unsigned(vm, "post-relax"); // default 0
    sD->endDislocationConfigurationPath = vm.raw("result-dislocation-configuration");
    sD->tau.reset(new AnalyticField());
    if (vm.has("no-external-stress") && vm.has("fixed-rate-external-stress"))
        die("Only one stress protocol can be defined at the same time!", -20);
    if (vm.has("fixed-rate-external-stress")) {
        std::unique_ptr<FixedRateProtocol> p;
        if (vm.has("spring-constant")) {
            std::unique_ptr<SpringProtocol> s(new SpringProtocol);
            s->setSpringConstant(as_double(vm, "spring-constant"));
            p.reset(s.release());
        } else {
            p.reset(new FixedRateProtocol);
        }
        p->setRate(as_double(vm, "fixed-rate-external-stress"));
        sD->externalStressProtocol.reset(p.release());
    } else {
        sD->externalStressProtocol.reset(new StressProtocol());
    }
    if (vm.has("change-cutoff-to-inf-under-threshold")) {
        sD->speedThresholdForCutoffChange = as_double(vm, "change-cutoff-to-inf-under-threshold");
        sD->isSpeedThresholdForCutoffChange = true;
    }
    return sD;
}

int as_int(const Values &v, const std::string &k)
{
    const std::string s = v.raw(k);
    char *end = nullptr;
    const long d = std::strtol(s.c_str(), &end, 10);
    if (s.empty() || *end != '\0' || d < -2147483648L || d > 2147483647L)
        die("the argument ('" + s + "') for option '--" + k + "' is invalid", -1);
    return (int)d;
}

// The eigenvalue analysis: processInput's EV branch (project_parser.cpp:299-318)
// and main (src/main.cpp:36-41).  getStressProtocol (:340-348) aborts unless a
// fixed-rate protocol is given, and is evaluated before getDataTimeSeries
// (:330-338) as GCC orders the constructor's arguments; getDataTimeSeries
// needs both the file list and the point-defect file (the reference then
// dereferences a null series; here that is an error exit).
int run_ev(const Values &vm)
{
    auto sD = std::make_shared<SimulationData>();
    if (!vm.count.count("result-ev-file") || vm.count.at("result-ev-file") != 1)
        die("result-ev-file is not defined! Exiting...", 1);
    sD->eVAnalResultFile = vm.raw("result-ev-file");
    if (vm.has("calculate-ev-deriv")) sD->calculateDerivativeEVAnal = true;
    sD->numberOfEigenVecToWrite = as_int(vm, "eigenvector-to-write"); // default 10
    if (vm.has("write-correlation-matrices")) sD->writeCorrelMatrices = as_int(vm, "write-correlation-matrices");
    if (!vm.has("fixed-rate-external-stress") || vm.count.at("fixed-rate-external-stress") != 1) {
        std::cerr << "the eigenvalue analysis needs --fixed-rate-external-stress" << std::endl;
        std::abort();
    }
    auto *protocol = new FixedRateProtocol;
    protocol->setRate(as_double(vm, "fixed-rate-external-stress"));
    std::unique_ptr<StressProtocol> owned(protocol);
    if (!vm.has("pd-configuration") || !vm.has("file-list") || vm.count.at("pd-configuration") != 1 ||
        vm.count.at("file-list") != 1)
        die("the eigenvalue analysis needs --file-list and --pd-configuration", 1);
    try {
        auto series = std::make_shared<DataTimeSeries>(vm.raw("file-list"), vm.raw("pd-configuration"));
        sdddstEV::TimeSeriesProcessor processor(sD, series, owned.release());
        processor.run();
    } catch (const EngineError &e) {
        std::cerr << "engine error " << e.code << ": " << e.what() << std::endl;
        return 3;
    } catch (const std::exception &e) {
        std::cerr << e.what() << std::endl;
        return 2;
    }
    return 0;
}

} // namespace

int main(int argc, char **argv)
{
    const Values vm = parse(argc, argv);
    if (!vm.has("hide-copyright"))
        std::cout << "sdddst_b200 - B200 engine for the SDDDST implicit step (drop-in for the sdddst simulation mode)\n";
    if (vm.has("help")) {
        print_help();
        return 0;
    }
    if (vm.has("ev-analyzation") && !vm.has("simulation")) return run_ev(vm);
    std::shared_ptr<SimulationData> sD = simulation_data(vm);
    try {
        Simulation simulation(sD);
        simulation.run();
    } catch (const EngineError &e) {
        std::cerr << "engine error " << e.code << ": " << e.what() << std::endl;
        return 3;
    }
    return 0;
}
