// Host C++ API of the engine: the reference's sdddstCore classes
// (Simulation, SimulationData, Field, AnalyticField, StressProtocol family,
// PrecisionHandler) with the same names and meaning, implemented on the C ABI
// of include/sdddst_b200.h.  Nothing here computes the physics on the CPU for
// a simulation: step(), calculateSpeeds(), calculateJacobian() and
// solveEQSys() run on the GPU; the host keeps the bookkeeping the reference
// keeps on the host (log lines, limits, avalanche counting, sub-configuration
// files).
#include "simulation.h"

#include "Fields/AnalyticField.h"
#include "Fields/PeriodicShearStressELTE.h"
#include "../../csrc/tabulated_field.cuh"
#include "Fields/PeriodicShearStressELTE.h"
#include "../../csrc/tabulated_field.cuh"
#include "StressProtocols/fixed_rate_protocol.h"
#include "StressProtocols/spring_protocol.h"
#include "constants.h"
#include "utility.h"

#include "../../../include/sdddst_b200.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <iomanip>
#include <sstream>

namespace sdddstCore {

// ------------------------------------------------------------------ Field

Field::Field() {}
Field::~Field() {}
double Field::xy(double, double) { return 0; }
double Field::xy_diff_x(double, double) { return 0; }
double Field::xy_diff_x2(double, double) { return 0; }
int Field::deviceKind() const { return -1; }

namespace {

// Image terms of the analytic field at separation (dx, dy): u_k = dx + k for
// the ten columns of AnalyticField::xy, cosh/sinh through E = e^{2 pi dx},
// the k = 0 column through 2(sinh^2 + sin^2) identities (no cancellation at
// small r).  Index order: 0 -> k=0, 1..4 -> +1..+4, 5..8 -> -1..-4, 9 -> end.
struct HostImages {
    double u[10], N[10], D[10], S[10], w[10], cy;
    bool pos;
};

void host_images(double dx, double dy, HostImages &im)
{
    const double sn = std::sin(M_PI * dy);
    const double sn2 = sn * sn;
    const double cy = 1.0 - 2.0 * sn2;
    const double em1 = std::expm1(M_PI * dx);
    const double ep = 1.0 + em1, E = ep * ep, Ei = 1.0 / E;
    const double sh = 0.5 * (em1 + em1 / ep), ch = 0.5 * (ep + 1.0 / ep);
    const double sh2 = sh * sh;
    im.cy = cy;
    im.pos = dx >= 0.0;
    im.u[0] = dx;
    im.D[0] = 2.0 * (sh2 + sn2);
    im.N[0] = 2.0 * (sh2 - sn2) - 4.0 * sh2 * sn2;
    im.S[0] = 2.0 * sh * ch;
    im.w[0] = 1.0;
    for (int k = 1; k <= 5; ++k) {
        const double q = std::exp(2.0 * M_PI * k), qi = 1.0 / q;
        if (k <= 4) {
            double a = E * q, b = Ei * qi, C = 0.5 * (a + b);
            im.u[k] = dx + k;
            im.N[k] = C * cy - 1.0;
            im.D[k] = C - cy;
            im.S[k] = 0.5 * (a - b);
            im.w[k] = 1.0;
            double c = E * qi, d = Ei * q, Cm = 0.5 * (c + d);
            im.u[4 + k] = dx - k;
            im.N[4 + k] = Cm * cy - 1.0;
            im.D[4 + k] = Cm - cy;
            im.S[4 + k] = 0.5 * (c - d);
            im.w[4 + k] = 1.0;
        } else {
            double a = im.pos ? E * qi : E * q, b = im.pos ? Ei * q : Ei * qi, C = 0.5 * (a + b);
            im.u[9] = im.pos ? dx - 5.0 : dx + 5.0;
            im.N[9] = C * cy - 1.0;
            im.D[9] = C - cy;
            im.S[9] = 0.5 * (a - b);
            im.w[9] = std::fabs(dx);
        }
    }
    im.w[4] = im.pos ? 1.0 - dx : 1.0;
    im.w[8] = im.pos ? 1.0 : 1.0 + dx;
}

const double kTwoPiSq = 2.0 * M_PI * M_PI;

} // namespace

AnalyticField::AnalyticField() : Field() {}
AnalyticField::~AnalyticField() {}
int AnalyticField::deviceKind() const { return SDDDST_FIELD_ANALYTIC; }

double AnalyticField::xy(double dx, double dy)
{
    HostImages im;
    host_images(dx, dy, im);
    double acc = 0.0;
    for (int k = 0; k < 10; ++k) acc += im.w[k] * im.u[k] * im.N[k] / (im.D[k] * im.D[k]);
    return acc * kTwoPiSq;
}

double AnalyticField::xy_diff_x(double dx, double dy)
{
    HostImages im;
    host_images(dx, dy, im);
    double acc = 0.0;
    for (int k = 0; k < 10; ++k) {
        const double r = 1.0 / im.D[k];
        acc += im.w[k] * r * r * (im.N[k] + 2.0 * M_PI * im.u[k] * im.S[k] * (im.cy - 2.0 * im.N[k] * r));
    }
    const int edge = im.pos ? 4 : 8;
    const double fe = im.u[9] * im.N[9] / (im.D[9] * im.D[9]);
    const double fg = im.u[edge] * im.N[edge] / (im.D[edge] * im.D[edge]);
    acc += im.pos ? fe - fg : fg - fe;
    return acc * kTwoPiSq;
}

double AnalyticField::xy_diff_x2(double dx, double dy)
{
    // fourth-order central difference of xy_diff_x (step 1e-4 |r| + 1e-7)
    const double r = std::sqrt(dx * dx + dy * dy);
    const double hh = 1e-4 * r + 1e-7;
    return (-xy_diff_x(dx + 2 * hh, dy) + 8 * xy_diff_x(dx + hh, dy) - 8 * xy_diff_x(dx - hh, dy) +
            xy_diff_x(dx - 2 * hh, dy)) /
           (12 * hh);
}

// --------------------------------------------------------- StressProtocol

StressProtocol::StressProtocol() {}
StressProtocol::~StressProtocol() {}
void StressProtocol::calculateStress(double, const std::vector<Dislocation> &, StressProtocolStepType) {}
double StressProtocol::getStress(StressProtocolStepType) { return 0; }
double StressProtocol::getStressDerivative(double) { return 0; }
bool StressProtocol::getTriggerState() { return false; }
std::string StressProtocol::getType() { return "zero-stress"; }
int StressProtocol::deviceKind() { return getType() == "zero-stress" ? SDDDST_STRESS_ZERO : -1; }

FixedRateProtocol::FixedRateProtocol() : StressProtocol(), rate(0), stressValues{0, 0, 0, 0} {}
FixedRateProtocol::~FixedRateProtocol() {}
void FixedRateProtocol::calculateStress(double t, const std::vector<Dislocation> &, StressProtocolStepType type)
{
    stressValues[(int)type] = t * rate;
}
double FixedRateProtocol::getStress(StressProtocolStepType type) { return stressValues[(int)type]; }
double FixedRateProtocol::getStressDerivative(double) { return rate; }
std::string FixedRateProtocol::getType() { return "fixed-rate-stress"; }
int FixedRateProtocol::deviceKind() { return SDDDST_STRESS_FIXED_RATE; }
double FixedRateProtocol::getRate() const { return rate; }
void FixedRateProtocol::setRate(double v) { rate = v; }

ConstantStressProtocol::ConstantStressProtocol(double v) : StressProtocol(), value(v) {}
double ConstantStressProtocol::getStress(StressProtocolStepType) { return value; }
std::string ConstantStressProtocol::getType() { return "constant-stress"; }
int ConstantStressProtocol::deviceKind() { return SDDDST_STRESS_CONSTANT; }
double ConstantStressProtocol::getValue() const { return value; }
void ConstantStressProtocol::setValue(double v) { value = v; }

SpringProtocol::SpringProtocol() : FixedRateProtocol(), springConstant(1.0) {}
SpringProtocol::~SpringProtocol() {}
void SpringProtocol::calculateStress(double t, const std::vector<Dislocation> &, StressProtocolStepType type,
                                     double strain)
{
    double v = springConstant * (t * rate - strain);
    stressValues[(int)type] = v < 0 ? 0 : v;
}
std::string SpringProtocol::getType() { return "spring-stress"; }
int SpringProtocol::deviceKind() { return SDDDST_STRESS_SPRING; }
double SpringProtocol::getSpringConstant() const { return springConstant; }
void SpringProtocol::setSpringConstant(double k) { springConstant = k; }

// ------------------------------------------------------ PrecisionHandler

PrecisionHandler::PrecisionHandler() : minPrecisity(1e-6), minPrecisitySqr(1e-12), maxErrorRatioSqr(0), selectedID(0) {}
PrecisionHandler::~PrecisionHandler() {}
void PrecisionHandler::setSize(unsigned int size) { toleranceAndError.resize(size, {minPrecisitySqr, 0.0}); }
unsigned long PrecisionHandler::getSize() const { return toleranceAndError.size(); }
void PrecisionHandler::reset()
{
    maxErrorRatioSqr = 0;
    for (auto &te : toleranceAndError) te = {minPrecisitySqr, 0.0};
}
void PrecisionHandler::updateTolerance(const double &d2, const unsigned int &id)
{
    const double t = d2 * 0.25 * 1e-2;
    if (t < minPrecisitySqr && t < toleranceAndError[id].first) toleranceAndError[id].first = t == 0.0 ? EPS : t;
}
void PrecisionHandler::updateError(const double &err, const unsigned int &id)
{
    if (toleranceAndError[id].second < err) {
        toleranceAndError[id].second = err;
        const double r = err * err / toleranceAndError[id].first;
        if (r > maxErrorRatioSqr) {
            maxErrorRatioSqr = r;
            selectedID = id;
        }
    }
}
double PrecisionHandler::getNewStepSize(const double &h) const
{
    if (maxErrorRatioSqr == 0.0) return 2.0 * h;
    double f = std::pow(1. / std::sqrt(maxErrorRatioSqr), 1. / 3.);
    return 0.9 * h * std::min(f, 2.0);
}
double PrecisionHandler::getMinPrecisity() const { return minPrecisity; }
void PrecisionHandler::setMinPrecisity(double v)
{
    minPrecisity = v;
    minPrecisitySqr = v * v;
}
double PrecisionHandler::getMaxErrorRatioSqr() const { return maxErrorRatioSqr; }
std::string PrecisionHandler::__str__() const
{
    return "N: " + std::to_string(toleranceAndError.size()) + " Prec: " + std::to_string(minPrecisity) +
           " New stepsize factor: " + std::to_string(getNewStepSize(1.0));
}
std::string PrecisionHandler::__repr__() const { return __str__(); }

// -------------------------------------------------------- SimulationData

SimulationData::SimulationData()
    : cutOffMultiplier(DEFAULT_CUTOFF_MULTIPLIER), cutOff(DEFAULT_CUTOFF), cutOffSqr(DEFAULT_CUTOFF * DEFAULT_CUTOFF),
      onePerCutOffSqr(1. / (DEFAULT_CUTOFF * DEFAULT_CUTOFF)), prec(DEFAULT_PRECISION), pc(0), dc(0),
      ic(DEFAULT_ITERATION_COUNT), timeLimit(DEFAULT_TIME_LIMIT), stepSize(DEFAULT_STEP_SIZE),
      simTime(DEFAULT_SIM_TIME), KASQR(DEFAULT_KASQR), A(DEFAULT_A), tau(nullptr), Ap(nullptr), Ai(nullptr),
      Ax(nullptr), x(nullptr), null(nullptr), Symbolic(nullptr), Numeric(nullptr), succesfulSteps(0),
      failedSteps(0), totalAccumulatedStrainIncrease(0), isStrainIncreaseLimit(false),
      totalAccumulatedStrainIncreaseLimit(0), isMaxStepSizeLimit(false), maxStepSizeLimit(0), isTimeLimit(false),
      isStepCountLimit(false), stepCountLimit(0), isSpeedLimit(false), finish(false), speedLimit(0),
      stressLimit(0), isStressLimit(false), calculateStrainDuringSimulation(false),
      orderParameterCalculationIsOn(false), endDislocationConfigurationPath(""), externalStressProtocol(nullptr),
      countAvalanches(false), avalancheSpeedThreshold(0), avalancheTriggerLimit(0), avalancheCount(0),
      inAvalanche(false), isSaveSubConfigs(false), subConfigPath(""), subConfigDelay(0),
      subConfigDelayDuringAvalanche(0), subconfigDistanceCounter(0), currentStressStateType(Original),
      speedThresholdForCutoffChange(0), isSpeedThresholdForCutoffChange(false), currentStorageSize(0),
      sumAvgSpeed(0), eVAnalResultFile(""), remainingFinalSteps(0), inFinal(false), calculateDerivativeEVAnal(false),
      numberOfEigenVecToWrite(10), writeCorrelMatrices(0), jacobianNonZeros(0)
{
}

SimulationData::SimulationData(const std::string &dconf, const std::string &pdconf) : SimulationData()
{
    readDislocationDataFromFile(dconf);
    readPointDefectDataFromFile(pdconf);
    initSimulationVariables();
}

SimulationData::~SimulationData() { releaseJacobian(); }

void SimulationData::releaseJacobian()
{
    std::free(Ap);
    std::free(Ai);
    std::free(Ax);
    std::free(x);
    Ap = Ai = nullptr;
    Ax = x = nullptr;
}

void SimulationData::resizeForDislocationCount()
{
    currentStorageSize = dc;
    for (auto *v : {&g, &initSpeed, &initSpeed2, &speed, &speed2, &dVec}) v->assign(dc, 0.0);
    bigStep.resize(dc);
    firstSmall.resize(dc);
    secondSmall.resize(dc);
    indexes.assign(dc, 0);
    releaseJacobian();
    x = static_cast<double *>(std::calloc(dc > 0 ? dc : 1, sizeof(double)));
}

// Text format of simulation_data.cpp:119-201: "x y b" (or "x y") per line.
void SimulationData::readDislocationDataFromFile(const std::string &path)
{
    if (path.empty()) return;
    std::ifstream in(path);
    if (!in.is_open()) throw std::runtime_error("cannot open dislocation data file: " + path);
    dislocations.clear();
    Dislocation d;
    while (in >> d.x >> d.y >> d.b) dislocations.push_back(d);
    dc = (unsigned)dislocations.size();
    resizeForDislocationCount();
}

void SimulationData::writeDislocationDataToFile(const std::string &path)
{
    std::ofstream out(path);
    if (!out.is_open()) throw std::runtime_error("cannot open the data file to write: " + path);
    out << std::scientific << std::setprecision(16);
    for (auto &d : dislocations) out << d.x << " " << d.y << " " << d.b << "\n";
}

void SimulationData::readPointDefectDataFromFile(const std::string &path)
{
    points.clear();
    pc = 0;
    if (path.empty()) return;
    std::ifstream in(path);
    if (!in.is_open()) throw std::runtime_error("cannot open point defect data file: " + path);
    PointDefect q;
    while (in >> q.x >> q.y) points.push_back(q);
    pc = (unsigned)points.size();
}

void SimulationData::writePointDefectDataToFile(const std::string &path)
{
    std::ofstream out(path);
    if (!out.is_open()) throw std::runtime_error("cannot open the data file to write: " + path);
    out << std::scientific << std::setprecision(16);
    for (auto &q : points) out << q.x << " " << q.y << "\n";
}

void SimulationData::initSimulationVariables() { updateCutOff(); }

// cutoff = m / sqrt(N), m -> 1e20 once m >= sqrt(2N)/12 (simulation_data.cpp:208-218)
void SimulationData::updateCutOff()
{
    double m = cutOffMultiplier;
    if (cutOffMultiplier >= 1. / 12. * std::sqrt(2.0 * double(dc))) m = 1e20;
    cutOff = 1. / std::sqrt(double(dc)) * m;
    cutOffSqr = cutOff * cutOff;
    onePerCutOffSqr = 1. / cutOffSqr;
}

// ------------------------------------------------------------ Simulation

static std::vector<double> pack(const std::vector<Dislocation> &d)
{
    std::vector<double> a(3 * d.size());
    for (size_t i = 0; i < d.size(); ++i) {
        a[3 * i] = d[i].x;
        a[3 * i + 1] = d[i].y;
        a[3 * i + 2] = d[i].b;
    }
    return a;
}

static void unpack(const std::vector<double> &a, std::vector<Dislocation> &d)
{
    d.resize(a.size() / 3);
    for (size_t i = 0; i < d.size(); ++i) d[i] = {a[3 * i], a[3 * i + 1], a[3 * i + 2]};
}

static bool same(const std::vector<Dislocation> &a, const std::vector<Dislocation> &b)
{
    if (a.size() != b.size()) return false;
    for (size_t i = 0; i < a.size(); ++i)
        if (a[i].x != b[i].x || a[i].y != b[i].y || a[i].b != b[i].b) return false;
    return true;
}

Simulation::Simulation(std::shared_ptr<SimulationData> _sD)
    : succesfulStep(true), lastWriteTimeFinished(0), initSpeedCalculationIsNeeded(true), firstStepRequest(true),
      energy(0), energyAccum(0), vsquare(0), sD(_sD), pH(new PrecisionHandler), ctx(nullptr),
      optPairsum(SDDDST_PAIRSUM_FP64), optSolver(SDDDST_SOLVER_GMRES_CLUSTER), optSolverTol(1e-13),
      pushedStep(0), pushedTime(0), stagedThisStep(false)
{
    sD->standardOutputLog << std::scientific << std::setprecision(16);
    pH->setMinPrecisity(sD->prec);
    pH->setSize(sD->dc);
}

Simulation::~Simulation()
{
    if (ctx) sdddst_ctx_destroy(ctx);
}

void Simulation::check(int rc)
{
    if (rc != SDDDST_OK) throw EngineError(rc, sdddst_last_error());
}

void Simulation::setEngineOptions(int pairsum, int solver, double solverTol)
{
    optPairsum = pairsum;
    optSolver = solver;
    optSolverTol = solverTol;
}

static void fill_params(SimulationData &sd, sdddst_params &p, int pairsum, int solver, double tol)
{
    sdddst_default_params(&p);
    p.n = (int)sd.dc;
    p.p = (int)sd.pc;
    p.cutoff_multiplier = sd.cutOffMultiplier;
    p.prec = sd.prec;
    p.step_size = sd.stepSize;
    p.A = sd.A;
    p.KASQR = sd.KASQR;
    p.ic = (int)sd.ic;
    p.calculate_strain = sd.calculateStrainDuringSimulation ? 1 : 0;
    p.max_step_limited = sd.isMaxStepSizeLimit ? 1 : 0;
    p.max_step = sd.maxStepSizeLimit;
    p.pairsum = pairsum;
    p.solver = solver;
    p.solver_tol = tol;
    if (!sd.tau) throw EngineError(SDDDST_ERR_INVALID, "SimulationData::tau is not set");
    p.field = sd.tau->deviceKind();
    if (p.field < 0) throw EngineError(SDDDST_ERR_INVALID, "the field has no device kernel (AnalyticField only)");
    StressProtocol *sp = sd.externalStressProtocol.get();
    if (!sp) throw EngineError(SDDDST_ERR_INVALID, "SimulationData::externalStressProtocol is not set");
    p.stress_kind = sp->deviceKind();
    if (p.stress_kind < 0) throw EngineError(SDDDST_ERR_INVALID, "the stress protocol has no device counterpart");
    if (auto *s = dynamic_cast<SpringProtocol *>(sp)) {
        p.stress_rate = s->getRate();
        p.spring_constant = s->getSpringConstant();
    } else if (auto *f = dynamic_cast<FixedRateProtocol *>(sp)) {
        p.stress_rate = f->getRate();
    } else if (auto *c = dynamic_cast<ConstantStressProtocol *>(sp)) {
        p.stress_value = c->getValue();
    }
}

void Simulation::ensureContext()
{
    if (ctx) return;
    sdddst_params p;
    fill_params(*sD, p, optPairsum, optSolver, optSolverTol);
    std::vector<double> xyb = pack(sD->dislocations), pd(2 * sD->points.size());
    for (size_t i = 0; i < sD->points.size(); ++i) {
        pd[2 * i] = sD->points[i].x;
        pd[2 * i + 1] = sD->points[i].y;
    }
    check(sdddst_ctx_create(&p, xyb.data(), pd.empty() ? nullptr : pd.data(), &ctx));
    pushed = sD->dislocations;
    pushedStep = sD->stepSize;
    pushedTime = sD->simTime;
}

// Brings the device up to date with anything the caller changed in
// SimulationData since the last step (configuration, step size, time,
// strain, cutoff multiplier, limits, protocol parameters).
void Simulation::pushState()
{
    ensureContext();
    sdddst_params p;
    fill_params(*sD, p, optPairsum, optSolver, optSolverTol);
    check(sdddst_update_params(ctx, &p));
    pH->setMinPrecisity(sD->prec);
    if (!same(pushed, sD->dislocations)) {
        std::vector<double> xyb = pack(sD->dislocations);
        check(sdddst_set_state(ctx, xyb.data(), sD->stepSize, sD->simTime, energy,
                               sD->totalAccumulatedStrainIncrease, firstStepRequest ? 1 : 0));
        pushed = sD->dislocations;
    } else {
        check(sdddst_set_scalars(ctx, sD->stepSize, sD->simTime, energy, sD->totalAccumulatedStrainIncrease));
    }
}

void Simulation::pullState()
{
    const size_t n = sD->dc;
    std::vector<double> buf(3 * n);
    std::vector<Dislocation> *cfg[] = {&sD->dislocations, &sD->bigStep, &sD->firstSmall, &sD->secondSmall};
    for (int w = 0; w < 4; ++w) {
        check(sdddst_get_config(ctx, w, buf.data()));
        unpack(buf, *cfg[w]);
    }
    std::vector<double> *vec[] = {&sD->initSpeed, &sD->initSpeed2, &sD->speed, &sD->speed2, &sD->dVec, &sD->g};
    for (int w = 0; w < 6; ++w) {
        vec[w]->resize(n);
        check(sdddst_get_vector(ctx, w, vec[w]->data()));
    }
    double sc[12];
    check(sdddst_get_scalars(ctx, sc));
    sD->simTime = sc[0];
    sD->stepSize = sc[1];
    sD->succesfulSteps = (size_t)sc[2];
    sD->failedSteps = (size_t)sc[3];
    energy = sc[4];
    sD->totalAccumulatedStrainIncrease = sc[5];
    sD->sumAvgSpeed = sc[7];
    vsquare = sc[8];
    energyAccum = sc[9];
    pushed = sD->dislocations;
}

std::vector<double> Simulation::lastTolerances()
{
    ensureContext();
    std::vector<double> t(sD->dc);
    check(sdddst_get_vector(ctx, 6, t.data()));
    return t;
}

double Simulation::lastMaxErrorRatioSqr()
{
    ensureContext();
    double sc[12];
    check(sdddst_get_scalars(ctx, sc));
    return sc[6];
}

// Simulation::step (simulation.cpp:435-441): the three stages run as one
// device step; the host then keeps the reference's bookkeeping.
bool Simulation::step()
{
    stepStageI();
    stepStageII();
    stepStageIII();
    return succesfulStep;
}

void Simulation::stepStageI()
{
    pushState();
    sD->currentStressStateType = Original;
    if (firstStepRequest && sD->standardOutputLog.is_open()) {
        // first log line (simulation.cpp:463-476) from the initial velocities
        StressProtocol *sp = sD->externalStressProtocol.get();
        if (auto *s = dynamic_cast<SpringProtocol *>(sp))
            s->calculateStress(sD->simTime, sD->dislocations, Original, sD->totalAccumulatedStrainIncrease);
        else
            sp->calculateStress(sD->simTime, sD->dislocations, Original);
        std::vector<double> v(sD->dc), m(sD->dc);
        std::vector<double> xyb = pack(sD->dislocations);
        check(sdddst_speeds_ext(ctx, xyb.data(), sp->getStress(Original), v.data(), m.data()));
        double sa = 0, sq = 0;
        for (double a : v) {
            sa += std::fabs(a);
            sq += a * a;
        }
        sD->standardOutputLog << sD->simTime << " " << sD->succesfulSteps << " " << sD->failedSteps << " " << 0
                              << " " << sa / double(sD->dc) << " " << sD->cutOff << " " << "-" << " "
                              << sp->getStress(Original) << " " << "-" << " " << sD->totalAccumulatedStrainIncrease
                              << " " << sq << " " << energy << "\n";
    }
    if (firstStepRequest) {
        lastWriteTimeFinished = get_wall_time();
        firstStepRequest = false;
        initSpeedCalculationIsNeeded = false;
    }
    int accepted = 0;
    check(sdddst_step(ctx, &accepted));
    succesfulStep = accepted != 0;
    stagedThisStep = true;
}

void Simulation::stepStageII()
{
    // the device step already ran both half steps in stepStageI
}

void Simulation::stepStageIII()
{
    if (!stagedThisStep) return;
    stagedThisStep = false;
    const double h_used = sD->stepSize;
    pullState();
    if (succesfulStep) afterAcceptedStep(h_used);
    if (sD->isMaxStepSizeLimit && sD->maxStepSizeLimit < sD->stepSize) sD->stepSize = sD->maxStepSizeLimit;
}

// Host bookkeeping of an accepted step (simulation.cpp:519-637).
void Simulation::afterAcceptedStep(double)
{
    if (sD->inFinal && sD->remainingFinalSteps > 0) sD->remainingFinalSteps--;
    StressProtocol *sp = sD->externalStressProtocol.get();
    if (auto *s = dynamic_cast<SpringProtocol *>(sp))
        s->calculateStress(sD->simTime, sD->dislocations, Original, sD->totalAccumulatedStrainIncrease);
    else
        sp->calculateStress(sD->simTime, sD->dislocations, Original);
    double orderParameter = sD->orderParameterCalculationIsOn ? calculateOrderParameter(sD->speed) : 0.0;
    const double now = get_wall_time();
    if (sD->sumAvgSpeed < sD->speedLimit && sD->isSpeedLimit) sD->finish = true;
    if (sD->countAvalanches) {
        if (sD->inAvalanche && sD->sumAvgSpeed < sD->avalancheSpeedThreshold) {
            sD->avalancheCount++;
            sD->inAvalanche = false;
        } else if (sD->sumAvgSpeed > sD->avalancheSpeedThreshold) {
            sD->inAvalanche = true;
        }
    }
    sD->standardOutputLog << sD->simTime << " " << sD->succesfulSteps << " " << sD->failedSteps << " "
                          << lastMaxErrorRatioSqr() << " " << sD->sumAvgSpeed << " " << sD->cutOff << " ";
    if (sD->orderParameterCalculationIsOn) sD->standardOutputLog << orderParameter;
    else sD->standardOutputLog << "-";
    sD->standardOutputLog << " " << sp->getStress(Original) << " " << now - lastWriteTimeFinished;
    if (sD->calculateStrainDuringSimulation) sD->standardOutputLog << " " << sD->totalAccumulatedStrainIncrease;
    else sD->standardOutputLog << " -";
    if (sD->isStressLimit && sp->getStress(Original) > sD->stressLimit) sD->finish = true;
    if (sD->isSpeedThresholdForCutoffChange && sD->speedThresholdForCutoffChange > sD->sumAvgSpeed) {
        sD->cutOffMultiplier = 1e20;
        sD->updateCutOff();
    }
    sD->standardOutputLog << " " << vsquare << " " << energy << "\n";
    if (sD->isSaveSubConfigs) {
        const bool due = (!sD->inAvalanche && sD->subConfigDelay >= sD->subconfigDistanceCounter) ||
                         (sD->inAvalanche && sD->subConfigDelayDuringAvalanche >= sD->subconfigDistanceCounter);
        if (due) {
            sD->subconfigDistanceCounter = 0;
            std::stringstream ss;
            ss << std::setprecision(16) << sD->simTime;
            sD->writeDislocationDataToFile(sD->subConfigPath + "/" + ss.str() + ".dconf");
        } else {
            sD->subconfigDistanceCounter++;
        }
    }
    lastWriteTimeFinished = get_wall_time();
}

// Simulation::run (simulation.cpp:417-433)
void Simulation::run()
{
    while (((sD->isTimeLimit && sD->simTime < sD->timeLimit) || !sD->isTimeLimit) &&
           ((sD->isStrainIncreaseLimit && sD->totalAccumulatedStrainIncrease < sD->totalAccumulatedStrainIncreaseLimit) ||
            !sD->isStrainIncreaseLimit) &&
           ((sD->isStepCountLimit && sD->succesfulSteps < sD->stepCountLimit) || !sD->isStepCountLimit) &&
           ((sD->countAvalanches && sD->avalancheCount < sD->avalancheTriggerLimit) || !sD->countAvalanches) &&
           !sD->finish)
        step();
    while (sD->remainingFinalSteps > 0) {
        sD->inFinal = true;
        step();
    }
    if (!sD->endDislocationConfigurationPath.empty()) sD->writeDislocationDataToFile(sD->endDislocationConfigurationPath);
}

double Simulation::getSimTime() { return sD->simTime; }
const std::vector<Dislocation> &Simulation::getStoredDislocationData() { return sD->dislocations; }

// calculateSpeeds (simulation.cpp:86-131) on the device; the stress of
// sD->currentStressStateType is added and the tolerances go to the host
// PrecisionHandler unless ignorePHUpdate.
void Simulation::calculateSpeeds(const std::vector<Dislocation> &dis, std::vector<double> &res, bool ignorePHUpdate)
{
    ensureContext();
    res.resize(dis.size());
    std::vector<double> m(dis.size());
    std::vector<double> xyb = pack(dis);
    const double tau = sD->externalStressProtocol->getStress(sD->currentStressStateType);
    check(sdddst_speeds_ext(ctx, xyb.data(), tau, res.data(), m.data()));
    if (!ignorePHUpdate)
        for (unsigned i = 0; i < dis.size(); ++i)
            if (std::isfinite(m[i])) pH->updateTolerance(m[i], i);
}

// calculateG (simulation.cpp:133-193)
void Simulation::calculateG(const double &stepsize, std::vector<Dislocation> &newDislocation,
                            const std::vector<Dislocation> &old, bool useSpeed2, bool calculateInitSpeed,
                            bool useInitSpeedForFirstStep, StressProtocolStepType origin, StressProtocolStepType end)
{
    std::vector<double> *isp = useSpeed2 ? &sD->initSpeed2 : &sD->initSpeed;
    std::vector<double> *csp = useSpeed2 ? &sD->speed2 : &sD->speed;
    StressProtocol *sp = sD->externalStressProtocol.get();
    auto set_stress = [&](double t, const std::vector<Dislocation> &d, StressProtocolStepType type, double strain) {
        if (auto *s = dynamic_cast<SpringProtocol *>(sp)) s->calculateStress(t, d, type, strain);
        else sp->calculateStress(t, d, type);
    };
    if (calculateInitSpeed) {
        double t = sD->simTime, tasi = sD->totalAccumulatedStrainIncrease;
        if (origin == EndOfFirstSmallStep) {
            t += sD->stepSize * 0.5;
            tasi += calculateStrainIncrement(sD->dislocations, sD->firstSmall);
        }
        set_stress(t, old, origin, tasi);
        sD->currentStressStateType = origin;
        calculateSpeeds(old, *isp);
    }
    if (useInitSpeedForFirstStep) {
        csp = isp;
    } else {
        double t = sD->simTime + sD->stepSize, tasi = sD->totalAccumulatedStrainIncrease;
        if (end == EndOfFirstSmallStep) {
            t -= sD->stepSize * 0.5;
            tasi += calculateStrainIncrement(sD->dislocations, sD->firstSmall);
        } else if (end == EndOfSecondSmallStep) {
            tasi += calculateStrainIncrement(sD->dislocations, sD->firstSmall) +
                    calculateStrainIncrement(sD->firstSmall, sD->secondSmall);
        } else if (end == EndOfBigStep) {
            tasi += calculateStrainIncrement(sD->dislocations, sD->bigStep);
        }
        set_stress(t, newDislocation, end, tasi);
        sD->currentStressStateType = end;
        calculateSpeeds(newDislocation, *csp);
    }
    sD->g.resize(sD->dc);
    for (size_t i = 0; i < sD->dc; ++i)
        sD->g[i] = newDislocation[i].x - (1.0 + sD->dVec[i]) * 0.5 * stepsize * (*csp)[i] - old[i].x -
                   (1.0 - sD->dVec[i]) * 0.5 * stepsize * (*isp)[i];
}

// calculateJacobian (simulation.cpp:236-384) on the device; the result is
// stored in the reference's CSC layout (Ap, Ai, Ax) with dVec and indexes.
void Simulation::calculateJacobian(const double &stepsize, const std::vector<Dislocation> &data)
{
    ensureContext();
    const int n = (int)sD->dc;
    std::vector<double> xyb = pack(data);
    std::vector<int> rp(n + 1);
    long nnz = 0;
    int rc = sdddst_jacobian(ctx, stepsize, xyb.data(), rp.data(), nullptr, nullptr, nullptr, 0, &nnz);
    if (rc != SDDDST_OK && rc != SDDDST_ERR_CAPACITY) check(rc);
    std::vector<int> col(nnz);
    std::vector<double> val(nnz);
    sD->dVec.resize(n);
    check(sdddst_jacobian(ctx, stepsize, xyb.data(), rp.data(), col.data(), val.data(), sD->dVec.data(), nnz, &nnz));
    // CSR of J -> CSC of J (rows ascending in each column)
    std::free(sD->Ap);
    std::free(sD->Ai);
    std::free(sD->Ax);
    sD->Ap = static_cast<int *>(std::calloc(n + 1, sizeof(int)));
    sD->Ai = static_cast<int *>(std::malloc(sizeof(int) * (nnz > 0 ? nnz : 1)));
    sD->Ax = static_cast<double *>(std::malloc(sizeof(double) * (nnz > 0 ? nnz : 1)));
    for (long q = 0; q < nnz; ++q) sD->Ap[col[q] + 1]++;
    for (int j = 0; j < n; ++j) sD->Ap[j + 1] += sD->Ap[j];
    std::vector<int> fill(sD->Ap, sD->Ap + n);
    for (int i = 0; i < n; ++i)
        for (int q = rp[i]; q < rp[i + 1]; ++q) {
            int p = fill[col[q]]++;
            sD->Ai[p] = i;
            sD->Ax[p] = val[q];
        }
    sD->indexes.assign(n, 0);
    for (int j = 0; j < n; ++j)
        for (int p = sD->Ap[j]; p < sD->Ap[j + 1]; ++p)
            if (sD->Ai[p] == j) sD->indexes[j] = p;
    sD->jacobianNonZeros = nnz;
}

void Simulation::calculateSparseFormForJacobian()
{
    // the device solve factors nothing up front; solveEQSys works on Ap/Ai/Ax
}

// solveEQSys (simulation.cpp:393-396): J x = g with J from Ap/Ai/Ax
void Simulation::solveEQSys()
{
    ensureContext();
    if (!sD->Ap) throw EngineError(SDDDST_ERR_INVALID, "no Jacobian: call calculateJacobian first");
    int it = 0;
    check(sdddst_solve_csc(ctx, sD->Ap, sD->Ai, sD->Ax, sD->g.data(), sD->x, &it));
}

// integrate (simulation.cpp:62-84) composed from the device operations above
void Simulation::integrate(const double &stepsize, std::vector<Dislocation> &newDislocation,
                           const std::vector<Dislocation> &old, bool useSpeed2, bool calculateInitSpeed,
                           StressProtocolStepType origin, StressProtocolStepType end)
{
    calculateJacobian(stepsize, newDislocation);
    calculateSparseFormForJacobian();
    const bool zero = sD->externalStressProtocol->getType() == "zero-stress";
    for (size_t i = 0; i < sD->ic; ++i) {
        if (i > 0) calculateG(stepsize, newDislocation, old, useSpeed2, false, false, origin, end);
        else calculateG(stepsize, newDislocation, old, useSpeed2, calculateInitSpeed, zero, origin, end);
        solveEQSys();
        for (size_t j = 0; j < sD->dc; ++j) newDislocation[j].x -= sD->x[j];
    }
}

// calculateXError (simulation.cpp:398-405) on the host PrecisionHandler
void Simulation::calculateXError()
{
    for (size_t i = 0; i < sD->dc; ++i) pH->updateError(std::fabs(sD->bigStep[i].x - sD->secondSmall[i].x), (unsigned)i);
}

double Simulation::calculateOrderParameter(const std::vector<double> &speeds)
{
    double s = 0;
    for (size_t i = 0; i < sD->dc && i < speeds.size(); ++i) s += sD->dislocations[i].b * speeds[i];
    return s;
}

// value stored at row j within [si, ei) of Ai/Ax (0 when absent), as
// getElement (simulation.cpp:195-229) answers it
double Simulation::getElement(int j, int si, int ei)
{
    int lo = si, hi = ei;
    while (lo < hi) {
        int mid = lo + (hi - lo) / 2;
        if (sD->Ai[mid] < j) lo = mid + 1;
        else hi = mid;
    }
    return (lo < ei && sD->Ai[lo] == j) ? sD->Ax[lo] : 0.0;
}

} // namespace sdddstCore

// ---------------------------------------------------------------- tabulated field
// Host tables of PeriodicShearStressELTE (the engine builds its own on the
// device): remainder of the analytic field after its image-free term.

namespace {

std::vector<double> build_remainder(bool dx_table)
{
    sdddstCore::AnalyticField af;
    auto rem = [&](double x, double y) {
        return dx_table ? af.xy_diff_x(x, y) - sd::tau0_xy_dx(x, y) : af.xy(x, y) - sd::tau0_xy(x, y);
    };
    std::vector<double> t((size_t)sd::kTabS * sd::kTabS);
    for (int ky = 0; ky < sd::kTabS; ++ky)
        for (int kx = 0; kx < sd::kTabS; ++kx) {
            const double x = sd::tab_coord(kx), y = sd::tab_coord(ky);
            double v;
            if (x == 0.0 && y == 0.0) { // limit at the origin: Richardson on symmetric averages
                auto avg = [&](double d) { return 0.25 * (rem(d, 0) + rem(-d, 0) + rem(0, d) + rem(0, -d)); };
                v = (4.0 * avg(1e-3) - avg(2e-3)) / 3.0;
            } else {
                v = rem(x, y);
            }
            t[(size_t)ky * sd::kTabS + kx] = v;
        }
    return t;
}

} // namespace

namespace sdddstCoreELTE {

PeriodicShearStressELTE::PeriodicShearStressELTE() : Field() {}
PeriodicShearStressELTE::~PeriodicShearStressELTE() {}
int PeriodicShearStressELTE::deviceKind() const { return SDDDST_FIELD_TABULATED; }

void PeriodicShearStressELTE::loadStress(std::string path, std::string type, int size)
{
    (void)path;
    if (size != sd::kTabG) throw std::invalid_argument("PeriodicShearStressELTE: tables are 1024 x 1024");
    if (type == "xy") remXY = build_remainder(false);
    else if (type == "xy_diff_x") remDX = build_remainder(true);
    else throw std::invalid_argument("PeriodicShearStressELTE: unknown table type " + type);
}

double PeriodicShearStressELTE::xy(double dx, double dy)
{
    if (remXY.empty()) throw std::logic_error("PeriodicShearStressELTE: call loadStress(path, \"xy\", 1024) first");
    normalize(dx);
    normalize(dy);
    return sd::tau0_xy(dx, dy) + sd::tab_interp(remXY.data(), dx, dy);
}

double PeriodicShearStressELTE::xy_diff_x(double dx, double dy)
{
    if (remDX.empty())
        throw std::logic_error("PeriodicShearStressELTE: call loadStress(path, \"xy_diff_x\", 1024) first");
    normalize(dx);
    normalize(dy);
    return sd::tau0_xy_dx(dx, dy) + sd::tab_interp(remDX.data(), dx, dy);
}

} // namespace sdddstCoreELTE
