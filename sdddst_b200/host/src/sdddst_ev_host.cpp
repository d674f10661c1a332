// Host side of the eigenvalue analysis: the reference's DataTimeSeries,
// sdddstEV::SpectralDecompositor and sdddstEV::TimeSeriesProcessor with the
// same names and meaning, on the engine's C ABI (sdddst_ev_analyze).  The
// Hessian, the eigenpairs, the observables, the derivatives and the
// correlation matrices are computed on the GPU; the host reads the files and
// writes the gzip text output in the reference's format
// (src/time_series_processor.cpp:21-204: std::ostream default formatting,
// values separated by single spaces).
#include "data_time_series.h"
#include "spectral_decompositor.h"
#include "time_series_processor.h"

#include "Fields/AnalyticField.h"
#include "StressProtocols/fixed_rate_protocol.h"
#include "constants.h"

#include "../../../include/sdddst_b200.h"

#include <zlib.h>

#include <algorithm>
#include <cmath>
#include <fstream>
#include <iostream>
#include <sstream>
#include <stdexcept>

namespace {

void check(int rc)
{
    if (rc != SDDDST_OK) throw sdddstCore::EngineError(rc, sdddst_last_error());
}

std::vector<double> pack(const std::vector<sdddstCore::Dislocation> &d)
{
    std::vector<double> xyb(3 * d.size());
    for (size_t i = 0; i < d.size(); ++i) {
        xyb[3 * i] = d[i].x;
        xyb[3 * i + 1] = d[i].y;
        xyb[3 * i + 2] = d[i].b;
    }
    return xyb;
}

std::vector<double> pack(const std::vector<sdddstCore::PointDefect> &p)
{
    std::vector<double> pd(2 * p.size());
    for (size_t i = 0; i < p.size(); ++i) {
        pd[2 * i] = p[i].x;
        pd[2 * i + 1] = p[i].y;
    }
    return pd;
}

// An engine context used for the analysis only: FP64 pair sums, the given
// velocity-side defect scaling and stress protocol.  The analysis has no
// cutoff; a cutoff multiplier of 1 keeps the context's Jacobian storage at the
// size of a sparse pattern.
void *analysis_ctx(const std::vector<double> &xyb, const std::vector<double> &pd, double A, double K,
                   int stress_kind, double rate)
{
    sdddst_params p;
    sdddst_default_params(&p);
    p.n = (int)(xyb.size() / 3);
    p.p = (int)(pd.size() / 2);
    p.cutoff_multiplier = 1.0;
    p.A = A;
    p.KASQR = K;
    p.stress_kind = stress_kind;
    p.stress_rate = rate;
    p.pairsum = SDDDST_PAIRSUM_FP64;
    void *ctx = nullptr;
    check(sdddst_ctx_create(&p, xyb.data(), pd.empty() ? nullptr : pd.data(), &ctx));
    return ctx;
}

} // namespace

// ------------------------------------------------------------ DataTimeSeries

// data_time_series.cpp:5-21: whitespace-separated "time path" pairs
DataTimeSeries::DataTimeSeries(std::string dconfList, std::string fconf) : fconfPath(fconf)
{
    std::ifstream dcs(dconfList);
    if (!dcs.is_open()) throw std::runtime_error("cannot open the file list: " + dconfList);
    std::string t, path;
    while (dcs >> t) {
        if (!(dcs >> path)) break;
        dconfs.push_back(std::make_pair(std::stod(t), path));
    }
}

// data_time_series.cpp:23-42
bool DataTimeSeries::next(std::shared_ptr<sdddstCore::SimulationData> sD)
{
    if (dconfs.empty()) return false;
    auto pair = dconfs.front();
    sD->readDislocationDataFromFile(pair.second);
    sD->readPointDefectDataFromFile(fconfPath);
    sD->A = DEFAULT_A * 1. / std::sqrt((double)sD->dc);
    sD->KASQR = DEFAULT_KASQR * double(sD->dc);
    sD->simTime = pair.first;
    dconfs.pop_front();
    return true;
}

namespace sdddstEV {

// ------------------------------------------------------ SpectralDecompositor

SpectralDecompositor::SpectralDecompositor(sdddstCore::Field *f)
    : dislocationCount(0), fpCount(0), field(f), ctx(nullptr)
{
}

SpectralDecompositor::~SpectralDecompositor()
{
    if (ctx) sdddst_ctx_destroy(ctx);
}

// spectral_decompositor.cpp:63-201 on the device: all n eigenpairs are read back
void SpectralDecompositor::decompose(std::vector<sdddstCore::Dislocation> &dislocations,
                                     std::vector<sdddstCore::PointDefect> &pointDefects)
{
    if (field && field->deviceKind() != SDDDST_FIELD_ANALYTIC)
        throw sdddstCore::EngineError(SDDDST_ERR_INVALID, "the eigenvalue analysis evaluates AnalyticField only");
    const std::vector<double> xyb = pack(dislocations), pd = pack(pointDefects);
    const int n = (int)dislocations.size();
    if (ctx && (dislocationCount != (unsigned long)n || pd != pdKey)) {
        sdddst_ctx_destroy(ctx);
        ctx = nullptr;
    }
    dislocationCount = n;
    fpCount = pointDefects.size();
    eigenValues.resize(n);
    vectors.assign((size_t)n * n, 0.0);
    if (n == 0) return;
    if (!ctx) {
        ctx = analysis_ctx(xyb, pd, DEFAULT_A, DEFAULT_KASQR, SDDDST_STRESS_ZERO, 0.0);
        pdKey = pd;
    }
    std::vector<double> w(n);
    check(sdddst_ev_analyze(ctx, xyb.data(), 0.0, w.data(), nullptr, nullptr, nullptr, nullptr, vectors.data(), n,
                            nullptr, nullptr, 0));
    for (int i = 0; i < n; ++i) eigenValues[i] = Pair{w[i], (unsigned long)i};
}

double SpectralDecompositor::getEigenValue(unsigned int i) { return eigenValues[i].eigen; }

double SpectralDecompositor::getEigenVectorElement(int i, int j)
{
    return vectors[eigenValues[i].index * dislocationCount + j];
}

unsigned long SpectralDecompositor::getDislocationCount() const { return dislocationCount; }
unsigned long SpectralDecompositor::getFpCount() const { return fpCount; }

// ------------------------------------------------------- TimeSeriesProcessor

TimeSeriesProcessor::TimeSeriesProcessor(std::shared_ptr<sdddstCore::SimulationData> _sD,
                                         std::shared_ptr<DataTimeSeries> dateTimeSeries,
                                         sdddstCore::StressProtocol *stressProtocol)
    : sD(_sD), dTS(dateTimeSeries), ctx(nullptr), ctxN(-1), ctxP(-1)
{
    sD->tau.reset(new sdddstCore::AnalyticField);
    sD->externalStressProtocol.reset(stressProtocol);
    sD->standardOutputLog = std::ofstream("/dev/null");
    sim.reset(new sdddstCore::Simulation(sD));
}

TimeSeriesProcessor::~TimeSeriesProcessor()
{
    if (ctx) sdddst_ctx_destroy(ctx);
}

// time_series_processor.cpp:21-204
void TimeSeriesProcessor::run()
{
    if (!dTS) throw sdddstCore::EngineError(SDDDST_ERR_INVALID, "no configuration series (file-list, pd-configuration)");
    gzFile out = gzopen(sD->eVAnalResultFile.c_str(), "wb");
    if (!out) throw std::runtime_error("cannot open the result file: " + sD->eVAnalResultFile);
    sdddstCore::StressProtocol *sp = sD->externalStressProtocol.get();
    const int kind = sp ? sp->deviceKind() : SDDDST_STRESS_ZERO;
    double rate = 0.0;
    if (auto *f = dynamic_cast<sdddstCore::FixedRateProtocol *>(sp)) rate = f->getRate();
    std::vector<double> pdKey;
    try {
        while (dTS->next(sD)) {
            if (sp) sp->calculateStress(sD->simTime, sD->dislocations, sdddstCore::StressProtocolStepType::Original);
            std::cout << sD->simTime << "\n";
            const int n = (int)sD->dc;
            const std::vector<double> xyb = pack(sD->dislocations), pd = pack(sD->points);
            if (ctx && (ctxN != n || pd != pdKey)) {
                sdddst_ctx_destroy(ctx);
                ctx = nullptr;
            }
            std::ostringstream line;
            line << sD->simTime;
            const int S = sD->writeCorrelMatrices;
            if (S < 0) throw sdddstCore::EngineError(SDDDST_ERR_INVALID, "write-correlation-matrices is negative");
            if (n > 0 && !ctx) {
                ctx = analysis_ctx(xyb, pd, sD->A, sD->KASQR, kind < 0 ? SDDDST_STRESS_ZERO : kind, rate);
                ctxN = n;
                ctxP = (int)sD->pc;
                pdKey = pd;
            }
            std::vector<double> ev(n), pn(n), gan(n), speeds(n), sums(n), deriv(n);
            const int nvec = S == 0 ? std::max(0, std::min(sD->numberOfEigenVecToWrite, n)) : 0;
            std::vector<double> vecs((size_t)nvec * n), corr(S > 0 ? (size_t)n * 3 * S * S : 0);
            const bool wantDeriv = S == 0 && sD->calculateDerivativeEVAnal;
            if (n > 0)
                check(sdddst_ev_analyze(ctx, xyb.data(), sD->simTime, ev.data(), pn.data(), sums.data(), gan.data(),
                                        speeds.data(), nvec ? vecs.data() : nullptr, nvec,
                                        wantDeriv ? deriv.data() : nullptr, S > 0 ? corr.data() : nullptr, S));
            for (int i = 0; i < n; ++i) line << " " << ev[i];
            for (int i = 0; i < n; ++i) line << " " << pn[i];
            for (int i = 0; i < n; ++i) line << " " << gan[i];
            if (S == 0) {
                for (int i = 0; i < n; ++i) line << " " << speeds[i];
                for (int i = 0; i < n; ++i) line << " " << sD->dislocations[i].x;
                for (int i = 0; i < n; ++i) line << " " << sums[i];
                for (int i = 0; i < nvec; ++i)
                    for (int j = 0; j < n; ++j) line << " " << vecs[(size_t)i * n + j];
                if (wantDeriv)
                    for (int i = 0; i < n; ++i) line << " " << deriv[i];
                line << "\n";
            } else {
                line << "\n";
                const size_t ss = (size_t)S * S;
                for (int m = 0; m < n; ++m)
                    for (int h = 0; h < 3; ++h) { // pp, pn, pppn
                        const double *c = corr.data() + ((size_t)m * 3 + h) * ss;
                        for (int i = 0; i < S; ++i) {
                            for (int j = 0; j < S; ++j) line << c[(size_t)i * S + j] << " ";
                            line << "\n";
                        }
                    }
            }
            const std::string s = line.str();
            for (size_t o = 0; o < s.size();) {
                const unsigned chunk = (unsigned)std::min<size_t>(s.size() - o, (size_t)1 << 30);
                if (gzwrite(out, s.data() + o, chunk) != (int)chunk)
                    throw std::runtime_error("writing the result file failed: " + sD->eVAnalResultFile);
                o += chunk;
            }
        }
    } catch (...) {
        gzclose(out);
        throw;
    }
    gzclose(out);
}

} // namespace sdddstEV
