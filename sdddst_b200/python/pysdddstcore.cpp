// PySdddstCore: the reference's Python module surface (src/bindings.cpp:49-210,
// python/src/*_wrapper.cpp) over the B200 engine's host API, with pybind11
// in place of Boost.Python (not installed).  Class, method and attribute
// names follow the reference so its README usage runs unchanged.
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>
#include <pybind11/stl_bind.h>

#include "Fields/AnalyticField.h"
#include "Fields/PeriodicShearStressELTE.h"
#include "StressProtocols/fixed_rate_protocol.h"
#include "StressProtocols/spring_protocol.h"
#include "simulation.h"
#include "utility.h"

#include <memory>
#include <string>

namespace py = pybind11;
using namespace sdddstCore;

PYBIND11_MAKE_OPAQUE(std::vector<Dislocation>)
PYBIND11_MAKE_OPAQUE(std::vector<PointDefect>)
PYBIND11_MAKE_OPAQUE(std::vector<double>)

namespace {

// Holder objects: init() creates the wrapped object, assigning it to a
// SimulationData transfers ownership and leaves the holder invalid
// (python/src/field_wrapper.cpp, stress_protocol_wrapper.cpp).
struct PyField {
    std::unique_ptr<Field> field;
    virtual ~PyField() {}
    virtual void init() { field.reset(new Field); }
    virtual std::string name() const { return "Field"; }
    bool valid() const { return field != nullptr; }
    std::string str() const { return name() + " - valid: " + (valid() ? "true" : "false"); }
};
struct PyAnalyticField : PyField {
    void init() override { field.reset(new AnalyticField); }
    std::string name() const override { return "AnalyticField"; }
};
// python/src/periodic_shear_stress_ELTE_wrapper.cpp:34-51
struct PyPeriodicShearStressFieldELTE : PyField {
    std::string pwd;
    void setPWD(std::string path) { pwd = path; }
    void init() override
    {
        std::unique_ptr<sdddstCoreELTE::PeriodicShearStressELTE> t(new sdddstCoreELTE::PeriodicShearStressELTE);
        t->loadStress(pwd, "xy", 1024);
        t->loadStress(pwd, "xy_diff_x", 1024);
        field.reset(t.release());
    }
    std::string name() const override { return "Periodic Shear Stress Field ELTE"; }
};
struct PyStressProtocol {
    std::unique_ptr<StressProtocol> protocol;
    virtual ~PyStressProtocol() {}
    virtual void init() { protocol.reset(new StressProtocol); }
    virtual std::string name() const { return "StressProtocol"; }
    bool valid() const { return protocol != nullptr; }
    std::string str() const { return name() + " - valid: " + (valid() ? "true" : "false"); }
};
struct PyFixedRateProtocol : PyStressProtocol {
    double rate = 0;
    void init() override
    {
        auto *p = new FixedRateProtocol;
        p->setRate(rate);
        protocol.reset(p);
    }
    std::string name() const override { return "FixedRateProtocol"; }
    double getRate() const { return rate; }
    void setRate(double r)
    {
        rate = r;
        if (auto *p = dynamic_cast<FixedRateProtocol *>(protocol.get())) p->setRate(r);
    }
};
struct PyConstantStressProtocol : PyStressProtocol {
    double value = 0;
    void init() override { protocol.reset(new ConstantStressProtocol(value)); }
    std::string name() const override { return "ConstantStressProtocol"; }
    double getValue() const { return value; }
    void setValue(double v)
    {
        value = v;
        if (auto *p = dynamic_cast<ConstantStressProtocol *>(protocol.get())) p->setValue(v);
    }
};
struct PySimulationData {
    std::shared_ptr<SimulationData> ptr;
    PySimulationData(const std::string &d, const std::string &p) : ptr(std::make_shared<SimulationData>(d, p)) {}
    SimulationData &resolve() { return *ptr; }
    std::string str() const
    {
        return "SimulationData N: " + std::to_string(ptr->dc) + " point defects: " + std::to_string(ptr->pc);
    }
};

double py_normalize(double v)
{
    normalize(v);
    return v;
}

} // namespace

PYBIND11_MODULE(PySdddstCore, m)
{
    m.doc() = "SDDDST implicit step on B200 (sm_100a): the PySdddstCore surface over the CUDA engine";
    m.def("hello_world", []() { return std::string("Hello World!"); });
    m.def("normalize", &py_normalize);
    m.def("X", &X);
    m.def("X2", &X2);
    m.def("E", &E);
    m.def("X_dx", &X_dx);
    m.def("X2_dx", &X2_dx);
    m.def("E_dx", &E_dx);
    m.def("get_wall_time", &get_wall_time);
    m.def("get_cpu_time", &get_cpu_time);

    py::class_<Dislocation>(m, "Dislocation")
        .def(py::init<>())
        .def(py::init([](double x, double y, double b) { return Dislocation{x, y, b}; }))
        .def_readwrite("x", &Dislocation::x)
        .def_readwrite("y", &Dislocation::y)
        .def_readwrite("b", &Dislocation::b)
        .def("__eq__", [](Dislocation &a, Dislocation b) { return a == b; })
        .def("__repr__", &Dislocation::__repr__)
        .def("__str__", &Dislocation::__str__);
    py::bind_vector<std::vector<Dislocation>>(m, "DislocationVector");
    py::class_<PointDefect>(m, "PointDefect")
        .def(py::init<>())
        .def(py::init([](double x, double y) { return PointDefect{x, y}; }))
        .def_readwrite("x", &PointDefect::x)
        .def_readwrite("y", &PointDefect::y)
        .def("__repr__", &PointDefect::__repr__)
        .def("__str__", &PointDefect::__str__);
    py::bind_vector<std::vector<PointDefect>>(m, "PointDefectVector");
    py::bind_vector<std::vector<double>>(m, "DoubleVector");

    py::class_<PrecisionHandler>(m, "PrecisionHandler")
        .def(py::init<>())
        .def("set_size", &PrecisionHandler::setSize)
        .def("get_size", &PrecisionHandler::getSize)
        .def("reset", &PrecisionHandler::reset)
        .def("update_tolerance", &PrecisionHandler::updateTolerance)
        .def("update_error", &PrecisionHandler::updateError)
        .def("get_new_stepsize", &PrecisionHandler::getNewStepSize)
        .def("get_min_precisity", &PrecisionHandler::getMinPrecisity)
        .def("set_min_precisity", &PrecisionHandler::setMinPrecisity)
        .def("get_max_error_ratio_square", &PrecisionHandler::getMaxErrorRatioSqr)
        .def("__repr__", &PrecisionHandler::__repr__)
        .def("__str__", &PrecisionHandler::__str__);

    py::class_<Field>(m, "Field")
        .def("xy", &Field::xy)
        .def("xy_diff_x", &Field::xy_diff_x)
        .def("xy_diff_x2", &Field::xy_diff_x2);
    py::class_<PyField>(m, "FieldObject")
        .def(py::init<>())
        .def("init", &PyField::init)
        .def("valid", &PyField::valid)
        .def("name", &PyField::name)
        .def("__str__", &PyField::str)
        .def("__repr__", &PyField::str);
    py::class_<PyAnalyticField, PyField>(m, "AnalyticFieldObject").def(py::init<>());
    py::class_<PyPeriodicShearStressFieldELTE, PyField>(m, "PeriodicShearStressFieldELTEObject")
        .def(py::init<>())
        .def("setPWD", &PyPeriodicShearStressFieldELTE::setPWD);

    py::enum_<StressProtocolStepType>(m, "StepType")
        .value("Original", Original)
        .value("EndOfBigStep", EndOfBigStep)
        .value("EndOfFirstSmallStep", EndOfFirstSmallStep)
        .value("EndOfSecondSmallStep", EndOfSecondSmallStep);
    py::class_<StressProtocol>(m, "StressProtocol")
        .def("calculate_stress", &StressProtocol::calculateStress)
        .def("get_stress", &StressProtocol::getStress)
        .def("get_type", &StressProtocol::getType);
    py::class_<PyStressProtocol>(m, "StressProtocolObject")
        .def(py::init<>())
        .def("init", &PyStressProtocol::init)
        .def("valid", &PyStressProtocol::valid)
        .def("name", &PyStressProtocol::name)
        .def("__repr__", &PyStressProtocol::str)
        .def("__str__", &PyStressProtocol::str);
    py::class_<PyFixedRateProtocol, PyStressProtocol>(m, "FixedRateStressProtocolObject")
        .def(py::init<>())
        .def_property("rate", &PyFixedRateProtocol::getRate, &PyFixedRateProtocol::setRate);
    py::class_<PyConstantStressProtocol, PyStressProtocol>(m, "ConstantStressProtocolObject")
        .def(py::init<>())
        .def_property("value", &PyConstantStressProtocol::getValue, &PyConstantStressProtocol::setValue);

    py::class_<SimulationData, std::shared_ptr<SimulationData>>(m, "SimulationData")
        .def(py::init<std::string, std::string>())
        .def("read_dislocation_data_from_file", &SimulationData::readDislocationDataFromFile)
        .def("write_dislocation_data_to_file", &SimulationData::writeDislocationDataToFile)
        .def("read_point_defect_data_from_file", &SimulationData::readPointDefectDataFromFile)
        .def("write_point_defect_data_to_file", &SimulationData::writePointDefectDataToFile)
        .def("init_simulation_variables", &SimulationData::initSimulationVariables)
        .def("update_cutoff", &SimulationData::updateCutOff)
        .def_readwrite("dislocations", &SimulationData::dislocations)
        .def_readwrite("point_defects", &SimulationData::points)
        .def_readwrite("g_vec", &SimulationData::g)
        .def_readwrite("init_speed", &SimulationData::initSpeed)
        .def_readwrite("init_speed_2", &SimulationData::initSpeed2)
        .def_readwrite("d_vec", &SimulationData::dVec)
        .def_readwrite("cutoff_multiplier", &SimulationData::cutOffMultiplier)
        .def_readwrite("cutoff", &SimulationData::cutOff)
        .def_readwrite("cutoff_square", &SimulationData::cutOffSqr)
        .def_readwrite("one_per_cutoff_square", &SimulationData::onePerCutOffSqr)
        .def_readwrite("precision", &SimulationData::prec)
        .def_readwrite("point_defect_count", &SimulationData::pc)
        .def_readwrite("dislocation_count", &SimulationData::dc)
        .def_readwrite("iteration_count", &SimulationData::ic)
        .def_readwrite("time_limit", &SimulationData::timeLimit)
        .def_readwrite("step_size", &SimulationData::stepSize)
        .def_readwrite("simulation_time", &SimulationData::simTime)
        .def_readwrite("KASQR", &SimulationData::KASQR)
        .def_readwrite("A", &SimulationData::A)
        .def_readwrite("big_step", &SimulationData::bigStep)
        .def_readwrite("first_small_step", &SimulationData::firstSmall)
        .def_readwrite("second_small_step", &SimulationData::secondSmall)
        .def_readwrite("successful_steps", &SimulationData::succesfulSteps)
        .def_readwrite("failed_steps", &SimulationData::failedSteps)
        .def_readwrite("total_accumulated_strain_increase", &SimulationData::totalAccumulatedStrainIncrease)
        .def_readwrite("strain_increase_limted", &SimulationData::isStrainIncreaseLimit)
        .def_readwrite("total_accumulated_strain_increase_limit",
                       &SimulationData::totalAccumulatedStrainIncreaseLimit)
        .def_readwrite("max_step_size_limited", &SimulationData::isMaxStepSizeLimit)
        .def_readwrite("max_stepsize_limit", &SimulationData::maxStepSizeLimit)
        .def_readwrite("time_limited", &SimulationData::isTimeLimit)
        .def_readwrite("step_count_limited", &SimulationData::isStepCountLimit)
        .def_readwrite("step_count_limit", &SimulationData::stepCountLimit)
        .def_readwrite("calculate_strain_during_simulation", &SimulationData::calculateStrainDuringSimulation)
        .def_readwrite("calculate_order_parameter", &SimulationData::orderParameterCalculationIsOn)
        .def_readwrite("final_dislocation_configuration_path", &SimulationData::endDislocationConfigurationPath)
        .def_readwrite("count_avalanches", &SimulationData::countAvalanches)
        .def_readwrite("avalanche_speed_threshold", &SimulationData::avalancheSpeedThreshold)
        .def_readwrite("trigger_limit_for_avalanche_count", &SimulationData::avalancheTriggerLimit)
        .def_readwrite("avalanche_count", &SimulationData::avalancheCount)
        .def_readwrite("in_avalanche", &SimulationData::inAvalanche)
        .def_readwrite("save_sub_configs", &SimulationData::isSaveSubConfigs)
        .def_readwrite("sub_config_path", &SimulationData::subConfigPath)
        .def_readwrite("sub_config_delay", &SimulationData::subConfigDelay)
        .def_readwrite("sub_config_delay_during_avalanche", &SimulationData::subConfigDelayDuringAvalanche)
        .def_readwrite("sub_config_distance_counter", &SimulationData::subconfigDistanceCounter)
        .def_readonly("stress_state", &SimulationData::currentStressStateType)
        .def_property(
            "tau", [](SimulationData &s) -> Field * { return s.tau.get(); },
            [](SimulationData &s, PyField &f) {
                if (f.valid()) s.tau.reset(f.field.release());
            },
            py::return_value_policy::reference_internal)
        .def_property(
            "external_stress", [](SimulationData &s) -> StressProtocol * { return s.externalStressProtocol.get(); },
            [](SimulationData &s, PyStressProtocol &p) {
                if (p.valid()) s.externalStressProtocol.reset(p.protocol.release());
            },
            py::return_value_policy::reference_internal);

    py::class_<PySimulationData>(m, "SimulationDataObject")
        .def(py::init<std::string, std::string>())
        .def("__call__", &PySimulationData::resolve, py::return_value_policy::reference_internal)
        .def("__repr__", &PySimulationData::str)
        .def("__str__", &PySimulationData::str);

    py::class_<Simulation>(m, "Simulation")
        .def_static(
            "create", [](PySimulationData &d) { return new Simulation(d.ptr); }, py::return_value_policy::take_ownership)
        .def("run", &Simulation::run)
        .def("step", &Simulation::step)
        .def("get_time", &Simulation::getSimTime)
        .def("set_engine_options", &Simulation::setEngineOptions)
        .def("last_tolerances", &Simulation::lastTolerances)
        .def("last_max_error_ratio_sqr", &Simulation::lastMaxErrorRatioSqr);
}
