/*
 * C harness around the reference hot path, compiled in place from the
 * reference sources (see oracle/Makefile).  Test infrastructure only: it is
 * the checker for the CUDA path, never part of the product.
 *
 * It builds a SimulationData exactly as the reference CLI does
 * (src/project_parser.cpp:137-298 of pgabor/sdddst): construct from the
 * dislocation/point-defect data, initSimulationVariables(), then the
 * initial step size, precision, cutoff multiplier + updateCutOff(), max step
 * size, the point-defect A/KASQR scaling (:208-212), strain/order-parameter
 * switches, tau = AnalyticField and the stress protocol.
 *
 * A "constant" stress protocol (getType() other than "zero-stress") is added
 * here because the reference has none; a fixed external stress of 0.01 is the
 * N=4096 workload's loading.
 *
 * Private members of Simulation / PrecisionHandler are read through a
 * `#define private public` applied to this translation unit only; the
 * reference objects themselves are compiled unmodified.  The per-step error
 * ratio and tolerance vector are captured by a link-time wrap of
 * PrecisionHandler::reset() (called once per step at src/simulation.cpp:644),
 * and the Jacobians / right-hand sides by the UMFPACK shim's recorder.
 */
#include <cmath>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <memory>
#include <numeric>
#include <sstream>
#include <string>
#include <vector>

#define private public
#define protected public
#include "simulation.h"
#include "simulation_data.h"
#include "precision_handler.h"
#include "Fields/AnalyticField.h"
#include "StressProtocols/stress_protocol.h"
#include "StressProtocols/fixed_rate_protocol.h"
#include "StressProtocols/spring_protocol.h"
#undef private
#undef protected

#include "spectral_decompositor.h"

#include "lapacke.h"
#include "umfpack.h"

using namespace sdddstCore;

namespace {

class ConstantStressProtocol : public StressProtocol
{
public:
    explicit ConstantStressProtocol(double v) : value(v) {}
    virtual double getStress(StressProtocolStepType) { return value; }
    virtual std::string getType() { return "constant-stress"; }
    double value;
};

struct Handle {
    std::shared_ptr<SimulationData> sd;
    std::unique_ptr<Simulation> sim;
    // captured by the reset() wrap
    double last_ratio = 0.0;
    std::vector<double> last_tol;
    int resets = 0;
};

Handle *g_active = nullptr;

} // namespace

extern "C" {

/* Parameters mirrored from the CLI (project_parser.cpp:39-94). */
typedef struct {
    double cutoff_multiplier; /* --cutoff-multiplier */
    double prec;              /* --position-precision */
    double step_size;         /* --initial-stepsize */
    int stress_kind;          /* 0 zero, 1 fixed-rate, 2 spring, 3 constant */
    double stress_rate;       /* --fixed-rate-external-stress */
    double spring_constant;   /* --spring-constant */
    double stress_value;      /* constant protocol value */
    int pd_scaling;           /* 1: A *= 1/sqrt(N), KASQR *= N (point-defect file given) */
    int calculate_strain;     /* --calculate-strain */
    int order_parameter;      /* --calculate-order-parameter */
    int max_step_limited;     /* --max-stepsize given */
    double max_step;
} ref_params;

/* PrecisionHandler::reset() wrap (linked with -Wl,--wrap=<mangled reset>). */
void __real__ZN10sdddstCore16PrecisionHandler5resetEv(PrecisionHandler *self);
void __wrap__ZN10sdddstCore16PrecisionHandler5resetEv(PrecisionHandler *self)
{
    if (g_active && g_active->sim && g_active->sim->pH.get() == self) {
        g_active->last_ratio = self->maxErrorRatioSqr;
        g_active->last_tol.resize(self->toleranceAndError.size());
        for (size_t i = 0; i < self->toleranceAndError.size(); ++i)
            g_active->last_tol[i] = self->toleranceAndError[i].first;
        g_active->resets++;
    }
    __real__ZN10sdddstCore16PrecisionHandler5resetEv(self);
}

static void load_dislocations(SimulationData &sd, int n, const double *xyb)
{
    sd.dislocations.resize(0);
    sd.dislocationDataIsLoaded = true;
    sd.dc = 0;
    for (int i = 0; i < n; ++i) {
        Dislocation d;
        d.x = xyb[3 * i];
        d.y = xyb[3 * i + 1];
        d.b = xyb[3 * i + 2];
        sd.dislocations.push_back(d);
        sd.dc++;
    }
    sd.updateMemoryUsageAccordingToDislocationCount();
}

static void load_points(SimulationData &sd, int p, const double *pd)
{
    sd.pc = 0;
    sd.points.resize(0);
    for (int i = 0; i < p; ++i) {
        PointDefect q;
        q.x = pd[2 * i];
        q.y = pd[2 * i + 1];
        sd.points.push_back(q);
        sd.pc++;
    }
}

void *ref_create(int n, const double *xyb, int p, const double *pd, const ref_params *prm)
{
    Handle *h = new Handle;
    h->sd = std::shared_ptr<SimulationData>(new SimulationData());
    SimulationData &sd = *h->sd;
    load_dislocations(sd, n, xyb);
    load_points(sd, p, pd);
    sd.initSimulationVariables();
    sd.stepSize = prm->step_size;
    sd.prec = prm->prec;
    sd.cutOffMultiplier = prm->cutoff_multiplier;
    sd.updateCutOff();
    if (prm->max_step_limited) {
        sd.maxStepSizeLimit = prm->max_step;
        sd.isMaxStepSizeLimit = true;
    }
    if (prm->pd_scaling) {
        sd.A *= 1. / sqrt(sd.dc);
        sd.KASQR *= double(sd.dc);
    }
    if (prm->calculate_strain) sd.calculateStrainDuringSimulation = true;
    if (prm->order_parameter) sd.orderParameterCalculationIsOn = true;
    sd.tau = std::unique_ptr<Field>(new AnalyticField());
    switch (prm->stress_kind) {
    case 1: {
        FixedRateProtocol *f = new FixedRateProtocol();
        f->setRate(prm->stress_rate);
        sd.externalStressProtocol = std::unique_ptr<StressProtocol>(f);
        break;
    }
    case 2: {
        SpringProtocol *s = new SpringProtocol();
        s->setSpringConstant(prm->spring_constant);
        s->setRate(prm->stress_rate);
        sd.externalStressProtocol = std::unique_ptr<StressProtocol>(s);
        break;
    }
    case 3:
        sd.externalStressProtocol = std::unique_ptr<StressProtocol>(new ConstantStressProtocol(prm->stress_value));
        break;
    default:
        sd.externalStressProtocol = std::unique_ptr<StressProtocol>(new StressProtocol());
    }
    h->sim = std::unique_ptr<Simulation>(new Simulation(h->sd));
    return h;
}

void ref_destroy(void *hp)
{
    Handle *h = (Handle *)hp;
    if (g_active == h) g_active = nullptr;
    delete h;
}

/* Scalars of SimulationData after construction:
 * out[0]=cutOff out[1]=cutOffSqr out[2]=onePerCutOffSqr out[3]=A out[4]=KASQR
 * out[5]=prec out[6]=stepSize out[7]=ic */
void ref_get_params(void *hp, double *out)
{
    Handle *h = (Handle *)hp;
    SimulationData &sd = *h->sd;
    out[0] = sd.cutOff;
    out[1] = sd.cutOffSqr;
    out[2] = sd.onePerCutOffSqr;
    out[3] = sd.A;
    out[4] = sd.KASQR;
    out[5] = sd.prec;
    out[6] = sd.stepSize;
    out[7] = sd.ic;
}

/* Simulation::step() (simulation.cpp:435).  Returns 1 on an accepted step. */
int ref_step(void *hp)
{
    Handle *h = (Handle *)hp;
    g_active = h;
    bool ok = h->sim->step();
    g_active = nullptr;
    return ok ? 1 : 0;
}

/* Step state after the last step:
 * out[0]=simTime out[1]=stepSize out[2]=succesfulSteps out[3]=failedSteps
 * out[4]=energy out[5]=totalAccumulatedStrainIncrease out[6]=maxErrorRatioSqr
 * (captured at the step's reset) out[7]=sumAvgSpeed out[8]=vsquare
 * out[9]=energyAccum out[10]=cutOff out[11]=stress(Original) */
void ref_get_scalars(void *hp, double *out)
{
    Handle *h = (Handle *)hp;
    SimulationData &sd = *h->sd;
    out[0] = sd.simTime;
    out[1] = sd.stepSize;
    out[2] = double(sd.succesfulSteps);
    out[3] = double(sd.failedSteps);
    out[4] = h->sim->energy;
    out[5] = sd.totalAccumulatedStrainIncrease;
    out[6] = h->last_ratio;
    out[7] = sd.sumAvgSpeed;
    out[8] = h->sim->vsquare;
    out[9] = h->sim->energyAccum;
    out[10] = sd.cutOff;
    out[11] = sd.externalStressProtocol->getStress(Original);
}

/* which: 0 dislocations, 1 bigStep, 2 firstSmall, 3 secondSmall -> N*3 */
void ref_get_config(void *hp, int which, double *xyb)
{
    Handle *h = (Handle *)hp;
    SimulationData &sd = *h->sd;
    const std::vector<Dislocation> *v = &sd.dislocations;
    if (which == 1) v = &sd.bigStep;
    if (which == 2) v = &sd.firstSmall;
    if (which == 3) v = &sd.secondSmall;
    for (size_t i = 0; i < v->size(); ++i) {
        xyb[3 * i] = (*v)[i].x;
        xyb[3 * i + 1] = (*v)[i].y;
        xyb[3 * i + 2] = (*v)[i].b;
    }
}

/* which: 0 initSpeed, 1 initSpeed2, 2 speed, 3 speed2, 4 dVec, 5 g,
 *        6 tolerance captured at the last step's reset */
void ref_get_vector(void *hp, int which, double *out)
{
    Handle *h = (Handle *)hp;
    SimulationData &sd = *h->sd;
    const std::vector<double> *v = &sd.initSpeed;
    if (which == 1) v = &sd.initSpeed2;
    if (which == 2) v = &sd.speed;
    if (which == 3) v = &sd.speed2;
    if (which == 4) v = &sd.dVec;
    if (which == 5) v = &sd.g;
    if (which == 6) v = &h->last_tol;
    for (size_t i = 0; i < v->size(); ++i) out[i] = (*v)[i];
}

/* Teacher forcing: restart from a given configuration, step size, time and
 * energy as if the previous step had just been accepted: initSpeed is
 * re-evaluated at the configuration (simulation.cpp:549) and the precision
 * handler is reset (:644), so the tolerance of the next step sees only that
 * step's own evaluations.  first_step=1 instead reproduces a fresh
 * Simulation's first step (:450-479). */
void ref_set_state(void *hp, const double *xyb, double step_size, double sim_time,
                   double energy, double strain, int first_step)
{
    Handle *h = (Handle *)hp;
    SimulationData &sd = *h->sd;
    for (size_t i = 0; i < sd.dislocations.size(); ++i) {
        sd.dislocations[i].x = xyb[3 * i];
        sd.dislocations[i].y = xyb[3 * i + 1];
        sd.dislocations[i].b = xyb[3 * i + 2];
    }
    sd.stepSize = step_size;
    sd.simTime = sim_time;
    sd.totalAccumulatedStrainIncrease = strain;
    h->sim->energy = energy;
    h->sim->pH->reset();
    if (first_step) {
        h->sim->firstStepRequest = true;
        h->sim->initSpeedCalculationIsNeeded = true;
        return;
    }
    h->sim->firstStepRequest = false;
    sd.currentStressStateType = Original;
    if (sd.externalStressProtocol->getType() == "spring-stress")
        static_cast<SpringProtocol *>(sd.externalStressProtocol.get())
            ->calculateStress(sd.simTime, sd.dislocations, Original, sd.totalAccumulatedStrainIncrease);
    else
        sd.externalStressProtocol->calculateStress(sd.simTime, sd.dislocations, Original);
    h->sim->calculateSpeeds(sd.dislocations, sd.initSpeed);
    h->sim->initSpeedCalculationIsNeeded = false;
    h->sim->pH->reset();
}

/* Simulation::calculateSpeeds (simulation.cpp:86) on a given configuration
 * with a fresh precision handler; returns velocities and per-dislocation
 * tolerances.  stress_type selects the StressProtocolStepType whose stored
 * stress value is added (after calculateStress(sim_time) for that type). */
void ref_speeds(void *hp, const double *xyb, double sim_time, int stress_type, double *v, double *tol)
{
    Handle *h = (Handle *)hp;
    SimulationData &sd = *h->sd;
    std::vector<Dislocation> dis(sd.dc);
    for (unsigned i = 0; i < sd.dc; ++i) {
        dis[i].x = xyb[3 * i];
        dis[i].y = xyb[3 * i + 1];
        dis[i].b = xyb[3 * i + 2];
    }
    StressProtocolStepType t = (StressProtocolStepType)stress_type;
    sd.externalStressProtocol->calculateStress(sim_time, dis, t);
    sd.currentStressStateType = t;
    h->sim->pH->reset();
    std::vector<double> res(sd.dc);
    h->sim->calculateSpeeds(dis, res);
    for (unsigned i = 0; i < sd.dc; ++i) {
        v[i] = res[i];
        tol[i] = h->sim->pH->toleranceAndError[i].first;
    }
    h->sim->pH->reset();
}

/* Simulation::calculateJacobian (simulation.cpp:236).  Copies the CSC
 * (column pointers Ap[N+1], row indices Ai[nnz], values Ax[nnz]) and dVec.
 * Returns nnz, or -(nnz) if cap is too small (nothing copied). */
long ref_jacobian(void *hp, double stepsize, const double *xyb, int *Ap, int *Ai, double *Ax,
                  double *dvec, long cap)
{
    Handle *h = (Handle *)hp;
    SimulationData &sd = *h->sd;
    std::vector<Dislocation> dis(sd.dc);
    for (unsigned i = 0; i < sd.dc; ++i) {
        dis[i].x = xyb[3 * i];
        dis[i].y = xyb[3 * i + 1];
        dis[i].b = xyb[3 * i + 2];
    }
    h->sim->calculateJacobian(stepsize, dis);
    long nnz = sd.Ap[sd.dc];
    if (nnz > cap) return -nnz;
    std::memcpy(Ap, sd.Ap, sizeof(int) * (sd.dc + 1));
    std::memcpy(Ai, sd.Ai, sizeof(int) * nnz);
    std::memcpy(Ax, sd.Ax, sizeof(double) * nnz);
    for (unsigned i = 0; i < sd.dc; ++i) dvec[i] = sd.dVec[i];
    return nnz;
}

/* One Simulation::integrate call (simulation.cpp:62) from the handle's
 * current state: stage 1 = big step (stepStageI's arguments), 2 = first small
 * step, 3 = second small step (requires stage 2 to have run).  Writes the
 * resulting configuration's x coordinates. */
void ref_integrate_stage(void *hp, int stage, double *x_out)
{
    Handle *h = (Handle *)hp;
    SimulationData &sd = *h->sd;
    Simulation &s = *h->sim;
    g_active = h;
    if (stage == 1) {
        sd.bigStep = sd.dislocations;
        s.integrate(sd.stepSize, sd.bigStep, sd.dislocations, false, s.initSpeedCalculationIsNeeded, Original, EndOfBigStep);
        for (unsigned i = 0; i < sd.dc; ++i) x_out[i] = sd.bigStep[i].x;
    } else if (stage == 2) {
        sd.firstSmall = sd.dislocations;
        s.integrate(0.5 * sd.stepSize, sd.firstSmall, sd.dislocations, false, false, Original, EndOfFirstSmallStep);
        for (unsigned i = 0; i < sd.dc; ++i) x_out[i] = sd.firstSmall[i].x;
    } else {
        sd.secondSmall = sd.firstSmall;
        s.integrate(0.5 * sd.stepSize, sd.secondSmall, sd.firstSmall, true, true, EndOfFirstSmallStep, EndOfSecondSmallStep);
        for (unsigned i = 0; i < sd.dc; ++i) x_out[i] = sd.secondSmall[i].x;
    }
    g_active = nullptr;
}

/* AnalyticField::xy / xy_diff_x / xy_diff_x2 (Fields/AnalyticField.cpp:145-202)
 * on arrays of separations. */
void ref_field(int which, long n, const double *dx, const double *dy, double *out)
{
    AnalyticField f;
    for (long i = 0; i < n; ++i) {
        if (which == 0) out[i] = f.xy(dx[i], dy[i]);
        else if (which == 1) out[i] = f.xy_diff_x(dx[i], dy[i]);
        else out[i] = f.xy_diff_x2(dx[i], dy[i]);
    }
}

/* SpectralDecompositor::decompose (src/spectral_decompositor.cpp:63-201) on
 * one configuration, through the LAPACKE shim: H = the matrix it hands to
 * LAPACKE_dsyevd (n x n), w = the eigenvalues it stores, V = eigenvector m at
 * V[m n ..] through getEigenVectorElement(m, j). */
void ref_ev_decompose(int n, const double *xyb, int p, const double *pd, double *H, double *w, double *V)
{
    std::vector<Dislocation> dis(n);
    std::vector<PointDefect> pts(p);
    for (int i = 0; i < n; ++i) dis[i] = Dislocation{xyb[3 * i], xyb[3 * i + 1], xyb[3 * i + 2]};
    for (int k = 0; k < p; ++k) pts[k] = PointDefect{pd[2 * k], pd[2 * k + 1]};
    sdddstEV::SpectralDecompositor dec(new AnalyticField);
    dec.decompose(dis, pts);
    lapacke_shim_last_input(H, (long)n * n);
    for (int m = 0; m < n; ++m) {
        w[m] = dec.getEigenValue(m);
        for (int j = 0; j < n; ++j) V[(size_t)m * n + j] = dec.getEigenVectorElement(m, j);
    }
}

} // extern "C"
