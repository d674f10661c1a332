// Step driver of the implicit scheme on the device (reference:
// src/simulation.cpp:62-84 integrate, :133-193 calculateG, :398-405
// calculateXError, :435-650 step / stepStageI-III; precision handler
// src/precision_handler.cpp:62-119; stress protocols
// src/StressProtocols/*.cpp; cutoff src/simulation_data.cpp:208-218).
//
// All vectors stay in HBM.  The host keeps the scalars the reference keeps
// in SimulationData / Simulation (step size, time, energy, counters, stress
// values) and issues the kernels on the context's stream.  Stage I and stage
// II share one Jacobian assembly: both are built at the accepted
// configuration, and H(h/2) = H(h)/2 exactly, so only d(h) differs.
#include "engine.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

namespace sd {

static const int kOrig = SDDDST_STAGE_ORIGINAL;
static const int kEndBig = SDDDST_STAGE_END_OF_BIG_STEP;
static const int kEndFirst = SDDDST_STAGE_END_OF_FIRST_SMALL_STEP;
static const int kEndSecond = SDDDST_STAGE_END_OF_SECOND_SMALL_STEP;

template <typename T>
static int dalloc(T **p, size_t count)
{
    if (count == 0) count = 1;
    return cudaMalloc((void **)p, sizeof(T) * count) == cudaSuccess ? 0 : SDDDST_ERR_NOMEM;
}

Engine::~Engine()
{
    if (device >= 0) cudaSetDevice(device);
    void *bufs[] = {d_x0, d_y, d_b, d_xb, d_x1, d_x2, d_xs, d_v0, d_v0b, d_vs, d_vs2, d_S0, d_S1, d_Stmp,
                    d_g, d_sol, d_dvec, d_tol, d_tol_last, d_minr2, d_part, d_pdx, d_pdy, d_cell,
                    d_cell_count, d_cell_start, d_cell_fill, d_sorted, d_rowcnt, d_rowptr, d_col, d_val,
                    d_V, d_w, d_z, d_r, d_hcol, d_partials, d_gs_partials, d_scal, d_y_small, d_ys, d_bs, d_flag, d_xw,
                    d_gdiag, d_valf, d_col_s, d_col_s16, d_vsort, d_xsrt, d_ysrt, d_bsrt, d_scan_tmp};
    for (void *b : bufs)
        if (b) cudaFree(b);
    if (h_scal) cudaFreeHost(h_scal);
    if (h_hrec) cudaFreeHost(h_hrec);
    if (d_hrec) cudaFree(d_hrec);
    if (d_counter) cudaFree(d_counter);
    precond_free(pc);
    precond_free(pc2);
    fused_free(*this);
    direct_free(*this);
    learned_free(*this);
    ev_free(*this);
    if (d_xasm) cudaFree(d_xasm);
    if (d_tol_snap) cudaFree(d_tol_snap);
    if (d_astat) cudaFree(d_astat);
    if (h_status) cudaFreeHost(h_status);
    if (d_tab_xy) cudaFree(d_tab_xy);
    if (d_tab_dx) cudaFree(d_tab_dx);
    if (st2) cudaStreamDestroy(st2);
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
    if (st) cudaStreamDestroy(st);
}

int Engine::side_streams()
{
    if (st2) return 0;
    if (cudaStreamCreateWithFlags(&st2, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming) != cudaSuccess) {
        err = "side stream creation failed";
        return SDDDST_ERR_CUDA;
    }
    return 0;
}

// The engine's launch functions all use `st`; exchanging it with st2 routes
// them to the side stream.
void Engine::fork_side()
{
    cudaEventRecord(ev_fork, st);
    cudaStreamWaitEvent(st2, ev_fork, 0);
    std::swap(st, st2);
}

void Engine::end_side()
{
    std::swap(st, st2);
    cudaEventRecord(ev_join, st2);
}

void Engine::join_side() { cudaStreamWaitEvent(st, ev_join, 0); }

int Engine::sync_check(const char *what)
{
    cudaError_t e1 = cudaStreamSynchronize(st);
    cudaError_t e2 = cudaGetLastError();
    cudaError_t e = e1 != cudaSuccess ? e1 : e2;
    if (e != cudaSuccess) {
        err = std::string(what) + ": " + cudaGetErrorString(e);
        return SDDDST_ERR_CUDA;
    }
    return 0;
}

// SimulationData::updateCutOff (simulation_data.cpp:208-218) and the cell
// grid of the neighbour search.
void Engine::update_cutoff()
{
    double m = cutoff_multiplier;
    if (cutoff_multiplier >= 1. / 12. * std::sqrt(2.0 * double(n))) m = 1e20;
    cutoff = 1. / std::sqrt((double)n) * m;
    cutoff_sqr = cutoff * cutoff;
    one_per_cutoff_sqr = 1. / cutoff_sqr;
    // pairs are kept while (r - c)^2 < 36.8 c^2, i.e. r < (1 + sqrt(36.8)) c
    double rc = cutoff * (1.0 + std::sqrt(36.8)) * (1.0 + 1e-9);
    int g = rc >= 1.0 / 3.0 ? 1 : (int)std::floor(1.0 / rc);
    if (g < 3) g = 1;
    if (g > 1024) g = 1024;
    G = g;
}

int Engine::init(const sdddst_params &p_, const double *xyb, const double *pd)
{
    prm = p_;
    n = prm.n;
    p = prm.p;
    device = prm.device;
    if (n < 2 || p < 0) {
        err = "n must be >= 2 and p >= 0";
        return SDDDST_ERR_INVALID;
    }
    if (!xyb || (p > 0 && !pd)) {
        err = "missing configuration arrays";
        return SDDDST_ERR_INVALID;
    }
    if (prm.ic < 1) prm.ic = 2;
    if (prm.gmres_restart < 2) prm.gmres_restart = 30;
    if (prm.gmres_restart > 31) prm.gmres_restart = 31; // fused Gram-Schmidt kernels hold 32 partial sums
    if (cudaSetDevice(device) != cudaSuccess) {
        err = "cudaSetDevice failed";
        return SDDDST_ERR_CUDA;
    }
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
        err = "stream creation failed";
        return SDDDST_ERR_CUDA;
    }
    cudaDeviceProp dp;
    cudaGetDeviceProperties(&dp, device);
    red_blocks = 2 * dp.multiProcessorCount;
    gs_blocks = dp.multiProcessorCount;
    cutoff_multiplier = prm.cutoff_multiplier;
    prec = prm.prec;
    A = prm.A;
    KASQR = prm.KASQR;
    ic = prm.ic;
    step_size = prm.step_size;
    restart = prm.gmres_restart;
    update_cutoff();

    int rc = 0;
    double **vecs[] = {&d_x0, &d_y, &d_b, &d_xb, &d_x1, &d_x2, &d_xs, &d_v0, &d_v0b, &d_vs, &d_vs2,
                       &d_S0, &d_S1, &d_Stmp, &d_g, &d_sol, &d_dvec, &d_tol, &d_tol_last, &d_w, &d_z,
                       &d_r, &d_ys, &d_bs, &d_xw, &d_gdiag, &d_vsort, &d_xsrt, &d_ysrt, &d_bsrt};
    for (double **v : vecs) rc |= dalloc(v, n);
    rc |= dalloc(&d_minr2, n);
    rc |= dalloc(&d_part, batch_backend ? 1 : pair_part_doubles(n));
    rc |= dalloc(&d_pdx, p);
    rc |= dalloc(&d_pdy, p);
    const int ncell = G * G;
    ncell_alloc = ncell;
    rc |= dalloc(&d_cell, n);
    rc |= dalloc(&d_cell_count, ncell + 1);
    rc |= dalloc(&d_cell_start, ncell + 1);
    rc |= dalloc(&d_cell_fill, ncell + 1);
    rc |= dalloc(&d_sorted, n);
    rc |= dalloc(&d_rowcnt, n);
    rc |= dalloc(&d_rowptr, n + 1);
    scan_tmp_cap = 2 * ((n + 2047) / 2048) + 2;
    rc |= dalloc(&d_scan_tmp, scan_tmp_cap);
    rc |= dalloc(&d_flag, 4);
    rc |= dalloc(&d_V, (size_t)(restart + 1) * n);
    rc |= dalloc(&d_hcol, 2 * (restart + 1) + 4);
    rc |= dalloc(&d_partials, (size_t)red_blocks * 32 + 64);
    rc |= dalloc(&d_gs_partials, (size_t)3 * gs_blocks * 32);
    coop_gs = gs_coop_supported(device, gs_blocks);
    rc |= dalloc(&d_hrec, (size_t)(restart + 1) * (2 * (restart + 1) + 1));
    rc |= dalloc(&d_counter, 4);
    if (cudaMallocHost((void **)&h_hrec, sizeof(double) * (restart + 1) * (2 * (restart + 1) + 1)) != cudaSuccess)
        rc |= SDDDST_ERR_NOMEM;
    rc |= dalloc(&d_scal, 8);
    rc |= dalloc(&d_y_small, (size_t)n + restart + 8);
    if (cudaMallocHost((void **)&h_scal, sizeof(double) * (2 * (restart + 1) + 8)) != cudaSuccess)
        rc |= SDDDST_ERR_NOMEM;
    rc |= precond_alloc(*this, pc);
    // the cluster solver runs device-resident on a single system (the CSR's
    // cell-sorted column positions are then always present)
    fused = prm.solver == SDDDST_SOLVER_GMRES_CLUSTER && std::getenv("SDDDST_HOST_GMRES") == nullptr;
    if (rc) {
        err = "device allocation failed";
        return SDDDST_ERR_NOMEM;
    }
    // initial CSR capacity from the expected neighbour count
    double rcut = cutoff * (1.0 + std::sqrt(36.8));
    double area = std::min(1.0, 3.14159265358979 * rcut * rcut);
    long est = (long)((double)n * (1.0 + 1.3 * area * n)) + n + 1024;
    if (est > (long)n * n + n) est = (long)n * n + n;
    nnz_cap = est;
    valf = prm.pairsum == SDDDST_PAIRSUM_FP32;
    rc |= alloc_csr_values(*this, nnz_cap);
    if (!rc) cudaMemsetAsync(d_col, 0, sizeof(int) * nnz_cap, st);
    if (rc) {
        err = "CSR allocation failed";
        return SDDDST_ERR_NOMEM;
    }
    // upload the configuration (AoS {x,y,b} -> SoA)
    std::vector<double> hx(n), hy(n), hb(n);
    for (int i = 0; i < n; ++i) {
        hx[i] = xyb[3 * i];
        hy[i] = xyb[3 * i + 1];
        hb[i] = xyb[3 * i + 2];
    }
    cudaMemcpyAsync(d_x0, hx.data(), sizeof(double) * n, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(d_y, hy.data(), sizeof(double) * n, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(d_b, hb.data(), sizeof(double) * n, cudaMemcpyHostToDevice, st);
    if (p > 0) {
        std::vector<double> px(p), py(p);
        for (int i = 0; i < p; ++i) {
            px[i] = pd[2 * i];
            py[i] = pd[2 * i + 1];
        }
        cudaMemcpyAsync(d_pdx, px.data(), sizeof(double) * p, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(d_pdy, py.data(), sizeof(double) * p, cudaMemcpyHostToDevice, st);
    }
    std::vector<double> t0(n, prec * prec);
    cudaMemcpyAsync(d_tol, t0.data(), sizeof(double) * n, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(d_tol_last, t0.data(), sizeof(double) * n, cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(d_dvec, 0, sizeof(double) * n, st);
    cudaMemsetAsync(d_counter, 0, sizeof(unsigned int), st);
    if (int rc = sync_check("init")) return rc;
    if (prm.field == SDDDST_FIELD_TABULATED) return tabulated_build(*this);
    return 0;
}

// ---------------------------------------------------------------- stress

void Engine::stress_calc(double t, int type, double strain_now)
{
    if (prm.stress_kind == SDDDST_STRESS_FIXED_RATE) {
        stress_vals[type] = t * prm.stress_rate; // fixed_rate_protocol.cpp:39-57
    } else if (prm.stress_kind == SDDDST_STRESS_SPRING) {
        double v = prm.spring_constant * (t * prm.stress_rate - strain_now); // spring_protocol.cpp:33-54
        if (v < 0) v = 0;
        stress_vals[type] = v;
    }
}

double Engine::stress_get(int type) const
{
    if (prm.stress_kind == SDDDST_STRESS_FIXED_RATE || prm.stress_kind == SDDDST_STRESS_SPRING)
        return stress_vals[type];
    if (prm.stress_kind == SDDDST_STRESS_CONSTANT) return prm.stress_value;
    return 0.0;
}

// ---------------------------------------------------------------- pieces

static void reset_tol(Engine &e)
{
    // PrecisionHandler::reset (precision_handler.cpp:62-70)
    std::vector<double> t0(e.n, e.prec * e.prec);
    cudaMemcpyAsync(e.d_tol, t0.data(), sizeof(double) * e.n, cudaMemcpyHostToDevice, e.st);
    cudaStreamSynchronize(e.st);
}

int Engine::speeds(const double *x, double *v_out, double *S_out, int stress_type, bool update_tol)
{
    const double tau_ext = stress_get(stress_type);
    const double r2_track = update_tol ? 400.0 * prec * prec * (1.0 + 1e-9) : 0.0;
    launch_pair_sum(*this, x, st, prm.pairsum, r2_track);
    launch_speeds_finish(*this, x, tau_ext, S_out, v_out, update_tol ? 1 : 0, st);
    launches += prm.pairsum == SDDDST_PAIRSUM_FP32 ? 4 : 3;
    return 0;
}

int Engine::assemble(const double *x)
{
    learned_invalidate(*this);
    pre_assembled = false;
    int rc = jacobian_assemble(*this, x);
    if (rc == 0 && (prm.solver == SDDDST_SOLVER_DIRECT || prm.solver == SDDDST_SOLVER_DIRECT_MIXED))
        rc = direct_analyse(*this, x);
    if (rc == 0 && (prm.solver == SDDDST_SOLVER_GMRES_LEARNED || prm.solver == SDDDST_SOLVER_GMRES_NEUMANN)) {
        if (!d_xasm && cudaMalloc(&d_xasm, sizeof(double) * n) != cudaSuccess) {
            err = "out of device memory";
            return SDDDST_ERR_NOMEM;
        }
        cudaMemcpyAsync(d_xasm, x, sizeof(double) * n, cudaMemcpyDeviceToDevice, st);
    }
    return rc;
}

// On a stall (no convergence within the iteration cap) the cluster
// preconditioner is rebuilt with a five times lower coupling threshold --
// larger clusters, more of the stiff couplings inverted exactly -- and the
// solve repeated, at most twice; the threshold returns to its setting for the
// next matrix.
int Engine::solve(double h, const double *rhs, double *x_out)
{
    if (prm.solver == SDDDST_SOLVER_DIRECT || prm.solver == SDDDST_SOLVER_DIRECT_MIXED)
        return direct_solve(*this, h, d_dvec, rhs, x_out);
    if (prm.solver == SDDDST_SOLVER_GMRES_LEARNED || prm.solver == SDDDST_SOLVER_GMRES_NEUMANN) {
        // GMRES preconditioned by B + C; on a stall, the device sparse LU of
        // the same matrix (analysed at the assembly positions)
        int rc = gmres_solve(*this, h, d_dvec, rhs, x_out, 4);
        if (rc != SDDDST_ERR_SOLVER) return rc;
        fallbacks++;
        if (int rc2 = direct_analyse(*this, d_xasm)) return rc2;
        if (int rc2 = direct_factor(*this, h, d_dvec)) return rc2;
        return direct_solve(*this, h, d_dvec, rhs, x_out);
    }
    if (prm.solver == SDDDST_SOLVER_GMRES_CLUSTER && fused && fused_supported(*this))
        return solve_fused(h, d_dvec, pc, rhs, x_out);
    int precond = prm.solver == SDDDST_SOLVER_GMRES_JACOBI ? 1 : prm.solver == SDDDST_SOLVER_GMRES_CLUSTER ? 2 : 0;
    int rc = gmres_solve(*this, h, d_dvec, rhs, x_out, precond);
    if (rc != SDDDST_ERR_SOLVER || precond != 2) return rc;
    const double theta0 = prm.precond_theta;
    for (int attempt = 0; attempt < 2 && rc == SDDDST_ERR_SOLVER; ++attempt) {
        prm.precond_theta = cluster_theta(*this) / 5.0;
        stalls++;
        if (int rc2 = precond_build(*this, h, d_dvec)) {
            prm.precond_theta = theta0;
            return rc2;
        }
        rc = gmres_solve(*this, h, d_dvec, rhs, x_out, precond);
    }
    if (prm.precond_theta != theta0) {
        prm.precond_theta = theta0;
        if (int rc2 = precond_build(*this, h, d_dvec)) return rc2;
    }
    return rc;
}

// One device-resident solve with the cluster preconditioner c of J(h); on a
// stall the preconditioner is rebuilt with a five times lower coupling
// threshold and the solve repeated, at most twice (as Engine::solve), and c
// is rebuilt at the setting afterwards.
int Engine::solve_fused(double h, const double *dvec, Cluster &c, const double *rhs, double *x_out)
{
    const Cluster *pcs[1] = {&c};
    int conv = 0;
    if (int rc = fused_gmres(*this, 1, &h, &dvec, &rhs, &x_out, pcs, &conv)) return rc;
    if (conv) return 0;
    const double theta0 = prm.precond_theta;
    for (int attempt = 0; attempt < 2 && !conv; ++attempt) {
        prm.precond_theta = cluster_theta(*this) / 5.0;
        stalls++;
        if (int rc = precond_build(*this, c, h, dvec)) {
            prm.precond_theta = theta0;
            return rc;
        }
        if (int rc = fused_gmres(*this, 1, &h, &dvec, &rhs, &x_out, pcs, &conv)) {
            prm.precond_theta = theta0;
            return rc;
        }
    }
    prm.precond_theta = theta0;
    if (int rc = precond_build(*this, c, h, dvec)) return rc;
    if (!conv) {
        err = "solve: GMRES did not reach the residual target";
        return SDDDST_ERR_SOLVER;
    }
    return 0;
}

int Engine::prepare_solver(double h, bool same_assembly)
{
    if (prm.solver == SDDDST_SOLVER_GMRES_CLUSTER) return precond_build(*this, h, d_dvec);
    if (prm.solver == SDDDST_SOLVER_DIRECT || prm.solver == SDDDST_SOLVER_DIRECT_MIXED)
        return direct_factor(*this, h, d_dvec);
    if (prm.solver == SDDDST_SOLVER_GMRES_LEARNED || prm.solver == SDDDST_SOLVER_GMRES_NEUMANN) {
        if (int rc = precond_build(*this, h, d_dvec)) return rc;
        // the network runs once per assembly: a second step size on the same
        // assembly (stage II's h/2 after stage I's h) rescales its outputs
        if (same_assembly && prm.solver == SDDDST_SOLVER_GMRES_LEARNED && learned_rescale(*this, h, d_dvec))
            return 0;
        // a new assembly right after an inference (stage III after stage I)
        // carries that inference's outputs onto its pattern
        if (!same_assembly && prm.solver == SDDDST_SOLVER_GMRES_LEARNED && learned_remap(*this, h, d_dvec))
            return 0;
        return learned_build(*this, h, d_dvec, d_xasm, prm.solver == SDDDST_SOLVER_GMRES_NEUMANN);
    }
    return 0;
}

int Engine::init_speeds(int origin, const double *xo, bool use2)
{
    double t = sim_time, tasi = strain;
    if (origin == kEndFirst) {
        t += step_size * 0.5;
        if (prm.stress_kind == SDDDST_STRESS_SPRING) {
            double inc;
            if (int rc = strain_inc(d_x0, d_x1, &inc)) return rc;
            tasi += inc;
        }
    }
    stress_calc(t, origin, tasi);
    cur_stress = origin;
    speeds(xo, use2 ? d_v0b : d_v0, use2 ? d_S1 : d_S0, origin, true);
    return 0;
}

// calculateG (simulation.cpp:133-193) of Newton iteration `it` of one stage.
int Engine::stage_residual(double h, int it, double *xn, const double *xo, bool use2, bool init_speed, int origin,
                           int end, double *csp0, const double *dvec, double *g)
{
    double *isp = use2 ? d_v0b : d_v0;
    const bool calc_init = it == 0 ? init_speed : false;
    const bool use_init_first = it == 0 ? zero_stress() : false;
    double *csp = csp0;
    if (calc_init)
        if (int rc = init_speeds(origin, xo, use2)) return rc;
    if (use_init_first) {
        csp = isp;
    } else {
        double t = sim_time + step_size, tasi = strain;
        if (prm.stress_kind == SDDDST_STRESS_SPRING) {
            double inc1 = 0, inc2 = 0;
            if (end == kEndFirst) {
                if (int rc = strain_inc(d_x0, d_x1, &inc1)) return rc;
            } else if (end == kEndSecond) {
                if (int rc = strain_inc(d_x0, d_x1, &inc1)) return rc;
                if (int rc = strain_inc(d_x1, d_x2, &inc2)) return rc;
            } else if (end == kEndBig) {
                if (int rc = strain_inc(d_x0, d_xb, &inc1)) return rc;
            }
            tasi += inc1 + inc2;
        }
        if (end == kEndFirst) t -= step_size * 0.5;
        stress_calc(t, end, tasi);
        cur_stress = end;
        speeds(xn, csp, d_Stmp, end, true);
    }
    launch_residual_g(*this, h, xn, xo, csp, isp, dvec, g, st);
    launches++;
    return 0;
}

// Simulation::integrate (simulation.cpp:62-84) with calculateG
// (simulation.cpp:133-193) inlined.
int Engine::integrate(double h, double *xn, const double *xo, bool use2, bool init_speed, int origin, int end,
                      bool reuse_assembly)
{
    if (!reuse_assembly)
        if (int rc = assemble(xn)) return rc;
    launch_make_dvec(*this, h, d_dvec, st);
    launches++;
    if (int rc = prepare_solver(h, reuse_assembly)) return rc;
    double *csp0 = use2 ? d_vs2 : d_vs;
    for (int it = 0; it < ic; ++it) {
        if (int rc = stage_residual(h, it, xn, xo, use2, init_speed, origin, end, csp0, d_dvec, d_g)) return rc;
        if (int rc = solve(h, d_g, d_sol)) return rc;
        launch_axpy_update(*this, xn, d_sol, st);
        launches++;
    }
    return 0;
}

// Stage I (integrate(h, bigStep, ...), simulation.cpp:443-492) and stage II
// (integrate(h/2, firstSmall, ...), :494-499) side by side: both start from
// the accepted configuration and share its assembly (H(h/2) = H(h)/2), and
// each chord-Newton iteration computes both residuals and then solves both
// systems in one device-resident launch that reads G once per SpMV pass.
// The order of the host-side stress evaluations, the velocity evaluations
// and the tolerance minimum is that of the two stages run one after the
// other, so the results are the same.  Stage I's current speed goes to its
// own buffer; stage II's to the speed vector the reference keeps.
int Engine::stages_one_two()
{
    if (int rc = fused_alloc(*this, 2)) {
        err = "fused solve: allocation failed";
        return rc;
    }
    const double h1 = step_size, h2 = 0.5 * step_size;
    if (int rc = assemble(d_xb)) return rc;
    launch_make_dvec(*this, h1, d_dvecI, st);
    launch_make_dvec(*this, h2, d_dvec, st);
    launches += 2;
    if (int rc = precond_build(*this, pc2, h1, d_dvecI, false)) return rc;
    if (int rc = precond_build(*this, pc, h2, d_dvec, false)) return rc;
    if (int rc = precond_check(*this, pc2)) return rc;
    if (int rc = precond_check(*this, pc)) return rc;
    for (int it = 0; it < ic; ++it) {
        if (int rc = stage_residual(h1, it, d_xb, d_x0, false, init_speed_needed, kOrig, kEndBig, d_vsI, d_dvecI,
                                    d_gI))
            return rc;
        if (int rc = stage_residual(h2, it, d_x1, d_x0, false, false, kOrig, kEndFirst, d_vs, d_dvec, d_g))
            return rc;
        const double hs[2] = {h1, h2};
        const double *dv[2] = {d_dvecI, d_dvec};
        const double *rhs[2] = {d_gI, d_g};
        double *xs[2] = {d_solI, d_sol};
        const Cluster *pcs[2] = {&pc2, &pc};
        int conv[2] = {0, 0};
        if (int rc = fused_gmres(*this, 2, hs, dv, rhs, xs, pcs, conv)) return rc;
        if (!conv[0])
            if (int rc = solve_fused(h1, d_dvecI, pc2, d_gI, d_solI)) return rc;
        if (!conv[1])
            if (int rc = solve_fused(h2, d_dvec, pc, d_g, d_sol)) return rc;
        launch_axpy_update(*this, d_xb, d_solI, st);
        launch_axpy_update(*this, d_x1, d_sol, st);
        launches += 2;
    }
    return 0;
}

// The three stages of an attempt with a wait at every check (assembly row
// counts, preconditioner builds, each solve): the path of every solver, and
// the fallback of an optimistic attempt that failed a check.
int Engine::stages_sync(double *ratio)
{
    const size_t bytes = sizeof(double) * n;
    cudaMemcpyAsync(d_xb, d_x0, bytes, cudaMemcpyDeviceToDevice, st);
    if (fused && prm.solver == SDDDST_SOLVER_GMRES_CLUSTER) {
        // ---- stages I and II together (one solve launch per Newton iteration)
        cudaMemcpyAsync(d_x1, d_x0, bytes, cudaMemcpyDeviceToDevice, st);
        if (int rc = stages_one_two()) return rc;
        successful_step = false;
    } else {
        if (int rc = integrate(step_size, d_xb, d_x0, false, init_speed_needed, kOrig, kEndBig, false)) return rc;
        successful_step = false;
        // ---- stage II (simulation.cpp:494-499): same configuration, same G
        cudaMemcpyAsync(d_x1, d_x0, bytes, cudaMemcpyDeviceToDevice, st);
        if (int rc = integrate(0.5 * step_size, d_x1, d_x0, false, false, kOrig, kEndFirst, true)) return rc;
    }
    // ---- stage III (simulation.cpp:501-650)
    sum_avg_speed = 0;
    cudaMemcpyAsync(d_x2, d_x1, bytes, cudaMemcpyDeviceToDevice, st);
    if (int rc = integrate(0.5 * step_size, d_x2, d_x1, true, true, kEndFirst, kEndSecond, false)) return rc;
    return stage_scalars(&vsquare1, &vsquare2, ratio);
}

// The three stages of an attempt of the device-resident cluster solver with
// no wait until they end: the assemblies do not read their row counts back
// (bounded by the CSR storage, guarded), the preconditioner builds and the
// solves leave their statuses on the device, and one copy after stage III
// brings back every status with |v0|^2, |v0b|^2 and the error ratio.  The
// work and its order are those of stages_sync.  *ok is false when a check
// failed (a stalled solve, a pattern larger than the storage, a
// non-finite Krylov quantity): the caller then redoes the attempt with waits,
// which repeats and reports the failure exactly as the waiting path does.
int Engine::stages_async(double *ratio, bool *ok)
{
    *ok = false;
    const size_t bytes = sizeof(double) * n;
    if (int rc = fused_alloc(*this, 2)) {
        err = "fused solve: allocation failed";
        return rc;
    }
    const double h1 = step_size, h2 = 0.5 * step_size;
    cudaMemcpyAsync(d_xb, d_x0, bytes, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(d_x1, d_x0, bytes, cudaMemcpyDeviceToDevice, st);
    // ---- stages I and II: shared assembly at the accepted configuration
    // (already built beside the previous attempt's last velocity evaluation
    // when that attempt was accepted)
    if (pre_assembled) {
        pre_assembled = false;
    } else {
        if (int rc = jacobian_assemble(*this, d_xb, true)) return rc;
        launch_csr_guard(*this, d_astat);
    }
    launch_make_dvec(*this, h1, d_dvecI, st);
    launch_make_dvec(*this, h2, d_dvec, st);
    launches += 2;
    if (int rc = precond_build(*this, pc2, h1, d_dvecI, false)) return rc;
    cudaMemcpyAsync(d_astat + 4, pc2.flag, sizeof(int), cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(d_astat + 5, pc2.bbase + n, sizeof(int), cudaMemcpyDeviceToDevice, st);
    if (int rc = precond_build(*this, pc, h2, d_dvec, false)) return rc;
    cudaMemcpyAsync(d_astat + 6, pc.flag, sizeof(int), cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(d_astat + 7, pc.bbase + n, sizeof(int), cudaMemcpyDeviceToDevice, st);
    for (int it = 0; it < ic; ++it) {
        if (int rc = stage_residual(h1, it, d_xb, d_x0, false, init_speed_needed, kOrig, kEndBig, d_vsI, d_dvecI,
                                    d_gI))
            return rc;
        if (int rc = stage_residual(h2, it, d_x1, d_x0, false, false, kOrig, kEndFirst, d_vs, d_dvec, d_g))
            return rc;
        const double hs[2] = {h1, h2};
        const double *dv[2] = {d_dvecI, d_dvec};
        const double *rhs[2] = {d_gI, d_g};
        double *xs[2] = {d_solI, d_sol};
        const Cluster *pcs[2] = {&pc2, &pc};
        if (int rc = fused_gmres(*this, 2, hs, dv, rhs, xs, pcs, nullptr, true, 2 * it)) return rc;
        launch_axpy_update(*this, d_xb, d_solI, st);
        launch_axpy_update(*this, d_x1, d_sol, st);
        launches += 2;
    }
    successful_step = false;
    // ---- stage III: assembly at the first small step's end
    sum_avg_speed = 0;
    cudaMemcpyAsync(d_x2, d_x1, bytes, cudaMemcpyDeviceToDevice, st);
    // the assembly, d and the preconditioner at the first small step's end on
    // the side stream, beside the velocity evaluation at the same
    // configuration (stage III's initial speeds) on the main stream
    fork_side();
    if (int rc = jacobian_assemble(*this, d_x2, true)) {
        end_side();
        return rc;
    }
    launch_csr_guard(*this, d_astat + 2);
    launch_make_dvec(*this, h2, d_dvec, st);
    launches++;
    if (int rc = precond_build(*this, pc, h2, d_dvec, false)) {
        end_side();
        return rc;
    }
    cudaMemcpyAsync(d_astat + 8, pc.flag, sizeof(int), cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(d_astat + 9, pc.bbase + n, sizeof(int), cudaMemcpyDeviceToDevice, st);
    end_side();
    if (int rc = init_speeds(kEndFirst, d_x1, true)) return rc;
    join_side();
    const int slot3 = 2 * ic;
    for (int it = 0; it < ic; ++it) {
        if (int rc = stage_residual(h2, it, d_x2, d_x1, true, false, kEndFirst, kEndSecond, d_vs2, d_dvec, d_g))
            return rc;
        const Cluster *pcs[1] = {&pc};
        const double *dv = d_dvec, *rhs = d_g;
        double *xs = d_sol;
        if (int rc = fused_gmres(*this, 1, &h2, &dv, &rhs, &xs, pcs, nullptr, true, slot3 + it)) return rc;
        launch_axpy_update(*this, d_x2, d_sol, st);
        launches++;
    }
    // ---- one copy of every status and the stage scalars, one wait
    launch_stage_scalars(*this);
    const int nslots = slot3 + ic;
    double *hs = h_status;
    cudaMemcpyAsync(hs, d_fstatus, sizeof(double) * 4 * nslots, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(hs + 4 * kAttemptSlots, d_scal, sizeof(double) * 3, cudaMemcpyDeviceToHost, st);
    int *ha = reinterpret_cast<int *>(hs + 4 * kAttemptSlots + 4);
    cudaMemcpyAsync(ha, d_astat, sizeof(int) * 10, cudaMemcpyDeviceToHost, st);
    if (int rc = sync_check("step")) return rc;
    // assemblies: a pattern beyond the storage grows it (the attempt is redone)
    for (int a = 0; a < 2; ++a) {
        const int total = ha[2 * a], flag = ha[2 * a + 1];
        if (flag == 1) {
            err = "jacobian: neighbour count and fill passes disagree";
            return SDDDST_ERR_CAPACITY;
        }
        if (flag == 2) {
            if (total < n) {
                err = "jacobian: row count overflow";
                return SDDDST_ERR_CAPACITY;
            }
            if (alloc_csr_values(*this, (long)total + total / 4 + 1024)) {
                err = "jacobian: CSR allocation failed";
                return SDDDST_ERR_NOMEM;
            }
            nnz_cap = (long)total + total / 4 + 1024;
            cudaMemsetAsync(d_col, 0, sizeof(int) * nnz_cap, st);
            return 0;
        }
    }
    nnz = ha[2];
    for (int b = 0; b < 3; ++b) {
        const int flag = ha[4 + 2 * b], nb = ha[5 + 2 * b];
        if (nb <= 0 || nb > n) {
            err = "precond: bad block count";
            return SDDDST_ERR_SOLVER;
        }
        if (flag) {
            err = "precond: singular cluster block";
            return SDDDST_ERR_SOLVER;
        }
    }
    long its = 0;
    for (int q = 0; q < nslots; ++q) {
        const double *sq = hs + 4 * q;
        if (sq[1] == 0.0 || sq[3] != 0.0) return 0; // a stall or a non-finite value: redo with waits
        its += (long)sq[0];
    }
    solves += nslots;
    iterations += its;
    last_iters = (int)hs[4 * (nslots - 1)];
    vsquare1 = hs[4 * kAttemptSlots];
    vsquare2 = hs[4 * kAttemptSlots + 1];
    *ratio = hs[4 * kAttemptSlots + 2];
    *ok = true;
    return 0;
}

// Simulation::step = stepStageI + II + III (simulation.cpp:435-650).
int Engine::step(int *accepted)
{
    const size_t bytes = sizeof(double) * n;
    // ---- stage I (simulation.cpp:443-492)
    energy_accum = 0;
    vsquare = 0;
    cur_stress = kOrig;
    if (first_step) {
        stress_calc(sim_time, kOrig, strain);
        speeds(d_x0, d_v0, d_S0, kOrig, true);
        init_speed_needed = false;
        if (int rc = sum_sq(d_v0, &vsquare)) return rc;
        first_step = false;
    }
    double ratio = 0.0;
    if (fused && prm.solver == SDDDST_SOLVER_GMRES_CLUSTER && ic <= 2) {
        if (!d_tol_snap) {
            if (cudaMalloc(&d_tol_snap, bytes) != cudaSuccess || cudaMalloc(&d_astat, sizeof(int) * 16) != cudaSuccess ||
                cudaMallocHost(&h_status, sizeof(double) * (4 * kAttemptSlots + 16)) != cudaSuccess) {
                err = "step: allocation failed";
                return SDDDST_ERR_NOMEM;
            }
        }
        if (int rc = side_streams()) return rc;
        cudaMemcpyAsync(d_tol_snap, d_tol, bytes, cudaMemcpyDeviceToDevice, st);
        bool ok = false;
        if (int rc = stages_async(&ratio, &ok)) return rc;
        if (!ok) {
            // a deferred check failed: the same attempt again, waiting at every check
            redone++;
            pre_assembled = false;
            cudaMemcpyAsync(d_tol, d_tol_snap, bytes, cudaMemcpyDeviceToDevice, st);
            if (int rc = stages_sync(&ratio)) return rc;
        }
    } else {
        if (int rc = stages_sync(&ratio)) return rc;
    }
    return finish_step(ratio, accepted);
}

// Error control, accept/reject and the new step size of an attempt
// (simulation.cpp:501-650, precision_handler.cpp:103-119).
int Engine::finish_step(double ratio, int *accepted)
{
    const size_t bytes = sizeof(double) * n;
    energy_accum = (vsquare1 + vsquare2) * 0.5 * step_size * 0.5;
    if (!std::isfinite(ratio)) {
        err = "step: non-finite error ratio";
        return SDDDST_ERR_NONFINITE;
    }
    if (ratio < 1.0) {
        successful_step = true;
        init_speed_needed = true;
        if (prm.calculate_strain) {
            double a, b2;
            if (int rc = strain_inc(d_x0, d_x1, &a)) return rc;
            strain += a;
            if (int rc = strain_inc(d_x1, d_x2, &b2)) return rc;
            strain += b2;
        }
        std::swap(d_x0, d_x2);
        sim_time += step_size;
        succ++;
        cur_stress = kOrig;
        stress_calc(sim_time, kOrig, strain);
        // the next attempt's stage I assembly at the new configuration on the
        // side stream, beside its velocity evaluation
        const bool pre = fused && prm.solver == SDDDST_SOLVER_GMRES_CLUSTER && ic <= 2 && st2;
        if (pre) {
            fork_side();
            const int rc = jacobian_assemble(*this, d_x0, true);
            if (rc == 0) launch_csr_guard(*this, d_astat);
            end_side();
            if (rc) return rc;
        }
        speeds(d_x0, d_v0, d_S0, kOrig, true);
        init_speed_needed = false;
        double sa, sq;
        if (int rc = abs_and_sq(d_v0, &sa, &sq)) return rc;
        if (pre) {
            // nothing stays in flight past the step: later calls may use the CSR
            if (cudaStreamSynchronize(st2) != cudaSuccess) return sync_check("side stream");
            pre_assembled = true;
        }
        sum_avg_speed = sa / double(n);
        vsquare = sq;
        energy_accum += (vsquare2 + vsquare) * 0.5 * step_size * 0.5;
        energy += energy_accum;
    } else {
        failed++;
    }
    // PrecisionHandler::getNewStepSize (precision_handler.cpp:103-119)
    double hn;
    if (0.0 == ratio) {
        hn = step_size * 2.0;
    } else {
        double t = 1. / std::sqrt(ratio);
        t = std::pow(t, 1. / 3.);
        if (t > 2.0) t = 2.0;
        hn = 0.9 * step_size * t;
    }
    step_size = hn;
    last_ratio = ratio;
    // PrecisionHandler::reset (precision_handler.cpp:62-70), kept for the
    // tolerance export
    cudaMemcpyAsync(d_tol_last, d_tol, bytes, cudaMemcpyDeviceToDevice, st);
    launch_fill(*this, d_tol, prec * prec);
    if (prm.max_step_limited && prm.max_step < step_size) step_size = prm.max_step;
    if (accepted) *accepted = successful_step ? 1 : 0;
    return sync_check("step");
}

int Engine::set_state_host(const double *xyb, double h, double t, double e, double s, int first)
{
    pre_assembled = false;
    std::vector<double> hx(n), hy(n), hb(n);
    for (int i = 0; i < n; ++i) {
        hx[i] = xyb[3 * i];
        hy[i] = xyb[3 * i + 1];
        hb[i] = xyb[3 * i + 2];
    }
    cudaMemcpyAsync(d_x0, hx.data(), sizeof(double) * n, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(d_y, hy.data(), sizeof(double) * n, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(d_b, hb.data(), sizeof(double) * n, cudaMemcpyHostToDevice, st);
    step_size = h;
    sim_time = t;
    strain = s;
    energy = e;
    reset_tol(*this);
    if (first) {
        first_step = true;
        init_speed_needed = true;
        return sync_check("set_state");
    }
    first_step = false;
    cur_stress = kOrig;
    stress_calc(sim_time, kOrig, strain);
    speeds(d_x0, d_v0, d_S0, kOrig, true);
    init_speed_needed = false;
    reset_tol(*this);
    return sync_check("set_state");
}

} // namespace sd
