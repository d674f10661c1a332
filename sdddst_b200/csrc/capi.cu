// extern "C" boundary of the engine (include/sdddst_b200.h).  Every entry
// point catches C++ exceptions and CUDA errors and turns them into status
// codes with a per-thread message.
#include "engine.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

namespace {

thread_local std::string g_last_error;

int fail(int rc, const std::string &msg)
{
    g_last_error = msg;
    return rc;
}

int from_engine(sd::Engine *e, int rc)
{
    if (rc != 0) g_last_error = e->err.empty() ? std::string("engine error") : e->err;
    return rc;
}

sd::Engine *E(void *ctx) { return static_cast<sd::Engine *>(ctx); }

// dst = src; *changed |= 1 where a bit pattern differs
__global__ void copy_compare_kernel(int n, const double *__restrict__ src, double *__restrict__ dst, int *changed)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double v = src[i];
    if (__double_as_longlong(v) != __double_as_longlong(dst[i])) atomicOr(changed, 1);
    dst[i] = v;
}

// Rejects a caller array holding NaN or Inf before anything reaches the
// device (the reference runs on with such values: a NaN velocity is accepted
// as a step and spreads through the configuration).  Returns 0 or
// SDDDST_ERR_NONFINITE with the first offending entry named.
int check_finite_f(const float *a, long count, const char *what)
{
    for (long k = 0; k < count; ++k)
        if (!std::isfinite(a[k]))
            return fail(SDDDST_ERR_NONFINITE, std::string(what) + ": non-finite value at index " + std::to_string(k));
    return 0;
}

int check_finite(const double *a, long count, const char *what)
{
    for (long k = 0; k < count; ++k)
        if (!std::isfinite(a[k]))
            return fail(SDDDST_ERR_NONFINITE, std::string(what) + ": non-finite value at index " + std::to_string(k));
    return 0;
}

// Uploads a caller configuration into the engine's scratch arrays and
// temporarily routes y and b to them; restores on destruction.
struct ScratchConfig {
    sd::Engine *e;
    double *y_saved, *b_saved;
    ScratchConfig(sd::Engine *e_, const double *xyb) : e(e_), y_saved(e_->d_y), b_saved(e_->d_b)
    {
        const int n = e->n;
        std::vector<double> hx(n), hy(n), hb(n);
        for (int i = 0; i < n; ++i) {
            hx[i] = xyb[3 * i];
            hy[i] = xyb[3 * i + 1];
            hb[i] = xyb[3 * i + 2];
        }
        cudaMemcpyAsync(e->d_xs, hx.data(), sizeof(double) * n, cudaMemcpyHostToDevice, e->st);
        cudaMemcpyAsync(e->d_ys, hy.data(), sizeof(double) * n, cudaMemcpyHostToDevice, e->st);
        cudaMemcpyAsync(e->d_bs, hb.data(), sizeof(double) * n, cudaMemcpyHostToDevice, e->st);
        cudaStreamSynchronize(e->st);
        e->d_y = e->d_ys;
        e->d_b = e->d_bs;
    }
    ~ScratchConfig()
    {
        e->d_y = y_saved;
        e->d_b = b_saved;
    }
};

} // namespace

namespace sd {
void set_last_error(const std::string &msg) { g_last_error = msg; }
} // namespace sd

extern "C" {

void sdddst_default_params(sdddst_params *p)
{
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->n = 0;
    p->p = 0;
    p->cutoff_multiplier = 1.0;           // DEFAULT_CUTOFF_MULTIPLIER, constants.h:26
    p->prec = 1e-8;                       // DEFAULT_PRECISION, constants.h:28
    p->step_size = 1.0;                   // DEFAULT_STEP_SIZE, constants.h:31
    p->A = 1e-4 * 16.0;                   // DEFAULT_A, constants.h:34
    p->KASQR = 1.65 * 1.65 * 1e6 / 256.0; // DEFAULT_KASQR, constants.h:33
    p->ic = 2;                            // DEFAULT_ITERATION_COUNT, constants.h:29
    p->stress_kind = SDDDST_STRESS_ZERO;
    p->spring_constant = 1.0;             // SpringProtocol(), spring_protocol.cpp:22-26
    p->field = SDDDST_FIELD_ANALYTIC;
    p->pairsum = SDDDST_PAIRSUM_FP64;
    p->solver = SDDDST_SOLVER_GMRES_CLUSTER;
    p->solver_tol = 1e-13;
    p->precond_theta = 0.0; // the solver's own default (cluster_theta)
    p->gmres_restart = 30;
    p->max_iters = 300;
    p->device = 0;
    p->neumann_theta = 0.0;
}

const char *sdddst_last_error(void) { return g_last_error.c_str(); }

int sdddst_ctx_create(const sdddst_params *prm, const double *xyb, const double *pd, void **ctx)
{
    if (!prm || !ctx) return fail(SDDDST_ERR_INVALID, "null argument");
    *ctx = nullptr;
    if (prm->field != SDDDST_FIELD_ANALYTIC && prm->field != SDDDST_FIELD_TABULATED)
        return fail(SDDDST_ERR_INVALID, "unsupported field kind");
    if (prm->pairsum != SDDDST_PAIRSUM_FP64 && prm->pairsum != SDDDST_PAIRSUM_FP32)
        return fail(SDDDST_ERR_INVALID, "unsupported pair-sum mode");
    if (prm->solver != SDDDST_SOLVER_GMRES && prm->solver != SDDDST_SOLVER_GMRES_JACOBI &&
        prm->solver != SDDDST_SOLVER_GMRES_CLUSTER && prm->solver != SDDDST_SOLVER_DIRECT &&
        prm->solver != SDDDST_SOLVER_GMRES_LEARNED && prm->solver != SDDDST_SOLVER_GMRES_NEUMANN &&
        prm->solver != SDDDST_SOLVER_DIRECT_MIXED)
        return fail(SDDDST_ERR_INVALID, "unsupported solver");
    if (!(prm->prec > 0) || !(prm->step_size > 0) || !(prm->cutoff_multiplier > 0))
        return fail(SDDDST_ERR_INVALID, "prec, step size and cutoff multiplier must be positive");
    if (xyb && prm->n > 0)
        if (int rc = check_finite(xyb, 3L * prm->n, "configuration")) return rc;
    if (pd && prm->p > 0)
        if (int rc = check_finite(pd, 2L * prm->p, "point defects")) return rc;
    sd::Engine *e = new (std::nothrow) sd::Engine();
    if (!e) return fail(SDDDST_ERR_NOMEM, "host allocation failed");
    int rc;
    try {
        rc = e->init(*prm, xyb, pd);
    } catch (const std::exception &ex) {
        rc = SDDDST_ERR_NOMEM;
        e->err = ex.what();
    }
    if (rc) {
        g_last_error = e->err;
        delete e;
        return rc;
    }
    *ctx = e;
    return SDDDST_OK;
}

int sdddst_ctx_destroy(void *ctx)
{
    if (!ctx) return SDDDST_OK;
    delete E(ctx);
    return SDDDST_OK;
}

int sdddst_set_state(void *ctx, const double *xyb, double step_size, double sim_time, double energy, double strain,
                     int first_step)
{
    if (!ctx || !xyb) return fail(SDDDST_ERR_INVALID, "null argument");
    if (!(step_size > 0)) return fail(SDDDST_ERR_INVALID, "step size must be positive");
    sd::Engine *e = E(ctx);
    if (int rc = check_finite(xyb, 3L * e->n, "configuration")) return rc;
    cudaSetDevice(e->device);
    try {
        return from_engine(e, e->set_state_host(xyb, step_size, sim_time, energy, strain, first_step));
    } catch (const std::exception &ex) {
        return fail(SDDDST_ERR_NOMEM, ex.what());
    }
}

int sdddst_get_scalars(void *ctx, double *out)
{
    if (!ctx || !out) return fail(SDDDST_ERR_INVALID, "null argument");
    sd::Engine *e = E(ctx);
    out[0] = e->sim_time;
    out[1] = e->step_size;
    out[2] = (double)e->succ;
    out[3] = (double)e->failed;
    out[4] = e->energy;
    out[5] = e->strain;
    out[6] = e->last_ratio;
    out[7] = e->sum_avg_speed;
    out[8] = e->vsquare;
    out[9] = e->energy_accum;
    out[10] = e->cutoff;
    out[11] = e->stress_get(SDDDST_STAGE_ORIGINAL);
    return SDDDST_OK;
}

int sdddst_get_config(void *ctx, int which, double *xyb)
{
    if (!ctx || !xyb || which < 0 || which > 3) return fail(SDDDST_ERR_INVALID, "bad argument");
    sd::Engine *e = E(ctx);
    cudaSetDevice(e->device);
    const int n = e->n;
    const double *src = which == 0 ? e->d_x0 : which == 1 ? e->d_xb : which == 2 ? e->d_x1 : e->d_x2;
    std::vector<double> hx(n), hy(n), hb(n);
    cudaMemcpyAsync(hx.data(), src, sizeof(double) * n, cudaMemcpyDeviceToHost, e->st);
    cudaMemcpyAsync(hy.data(), e->d_y, sizeof(double) * n, cudaMemcpyDeviceToHost, e->st);
    cudaMemcpyAsync(hb.data(), e->d_b, sizeof(double) * n, cudaMemcpyDeviceToHost, e->st);
    if (int rc = e->sync_check("get_config")) return from_engine(e, rc);
    for (int i = 0; i < n; ++i) {
        xyb[3 * i] = hx[i];
        xyb[3 * i + 1] = hy[i];
        xyb[3 * i + 2] = hb[i];
    }
    return SDDDST_OK;
}

int sdddst_get_vector(void *ctx, int which, double *out)
{
    if (!ctx || !out || which < 0 || which > 6) return fail(SDDDST_ERR_INVALID, "bad argument");
    sd::Engine *e = E(ctx);
    cudaSetDevice(e->device);
    const double *src[] = {e->d_v0, e->d_v0b, e->d_vs, e->d_vs2, e->d_dvec, e->d_g, e->d_tol_last};
    cudaMemcpyAsync(out, src[which], sizeof(double) * e->n, cudaMemcpyDeviceToHost, e->st);
    return from_engine(e, e->sync_check("get_vector"));
}

int sdddst_speeds(void *ctx, const double *xyb, double sim_time, int stress_type, double *v, double *tol)
{
    if (!ctx || !xyb || !v || !tol || stress_type < 0 || stress_type > 3)
        return fail(SDDDST_ERR_INVALID, "bad argument");
    sd::Engine *e = E(ctx);
    if (int rc = check_finite(xyb, 3L * e->n, "configuration")) return rc;
    cudaSetDevice(e->device);
    try {
        ScratchConfig sc(e, xyb);
        e->stress_calc(sim_time, stress_type, e->strain);
        std::vector<double> t0(e->n, e->prec * e->prec);
        // fresh precision handler for this evaluation
        cudaMemcpyAsync(e->d_tol_last, e->d_tol, sizeof(double) * e->n, cudaMemcpyDeviceToDevice, e->st);
        cudaMemcpyAsync(e->d_tol, t0.data(), sizeof(double) * e->n, cudaMemcpyHostToDevice, e->st);
        e->speeds(e->d_xs, e->d_Stmp + 0, e->d_w, stress_type, true);
        cudaMemcpyAsync(v, e->d_Stmp, sizeof(double) * e->n, cudaMemcpyDeviceToHost, e->st);
        cudaMemcpyAsync(tol, e->d_tol, sizeof(double) * e->n, cudaMemcpyDeviceToHost, e->st);
        cudaMemcpyAsync(e->d_tol, e->d_tol_last, sizeof(double) * e->n, cudaMemcpyDeviceToDevice, e->st);
        return from_engine(e, e->sync_check("speeds"));
    } catch (const std::exception &ex) {
        return fail(SDDDST_ERR_NOMEM, ex.what());
    }
}

int sdddst_speeds_ext(void *ctx, const double *xyb, double tau_ext, double *v, double *minr2)
{
    if (!ctx || !xyb || !v) return fail(SDDDST_ERR_INVALID, "bad argument");
    sd::Engine *e = E(ctx);
    if (int rc = check_finite(xyb, 3L * e->n, "configuration")) return rc;
    cudaSetDevice(e->device);
    try {
        ScratchConfig sc(e, xyb);
        const double r2_track = 400.0 * e->prec * e->prec * (1.0 + 1e-9);
        sd::launch_pair_sum(*e, e->d_xs, e->st, e->prm.pairsum, r2_track);
        e->d_minr2_out = e->d_z;
        sd::launch_speeds_finish(*e, e->d_xs, tau_ext, nullptr, e->d_Stmp, 0, e->st);
        e->d_minr2_out = nullptr;
        e->launches += e->prm.pairsum == SDDDST_PAIRSUM_FP32 ? 4 : 3;
        cudaMemcpyAsync(v, e->d_Stmp, sizeof(double) * e->n, cudaMemcpyDeviceToHost, e->st);
        if (minr2) cudaMemcpyAsync(minr2, e->d_z, sizeof(double) * e->n, cudaMemcpyDeviceToHost, e->st);
        return from_engine(e, e->sync_check("speeds_ext"));
    } catch (const std::exception &ex) {
        return fail(SDDDST_ERR_NOMEM, ex.what());
    }
}

int sdddst_set_scalars(void *ctx, double step_size, double sim_time, double energy, double strain)
{
    if (!ctx) return fail(SDDDST_ERR_INVALID, "null argument");
    if (!(step_size > 0)) return fail(SDDDST_ERR_INVALID, "step size must be positive");
    sd::Engine *e = E(ctx);
    e->step_size = step_size;
    e->sim_time = sim_time;
    e->energy = energy;
    e->strain = strain;
    return SDDDST_OK;
}

int sdddst_update_params(void *ctx, const sdddst_params *prm)
{
    if (!ctx || !prm) return fail(SDDDST_ERR_INVALID, "null argument");
    sd::Engine *e = E(ctx);
    e->pre_assembled = false; // the stored pattern no longer matches the next attempt
    if (prm->n != e->n || prm->p != e->p || prm->field != e->prm.field || prm->pairsum != e->prm.pairsum)
        return fail(SDDDST_ERR_INVALID, "sizes, field and pair-sum mode cannot change on a live context");
    if (!(prm->prec > 0) || !(prm->cutoff_multiplier > 0)) return fail(SDDDST_ERR_INVALID, "bad parameter");
    cudaSetDevice(e->device);
    const int restart_alloc = e->restart;
    e->prm.cutoff_multiplier = prm->cutoff_multiplier;
    e->prm.prec = prm->prec;
    e->prm.max_step_limited = prm->max_step_limited;
    e->prm.max_step = prm->max_step;
    e->prm.stress_kind = prm->stress_kind;
    e->prm.stress_rate = prm->stress_rate;
    e->prm.spring_constant = prm->spring_constant;
    e->prm.stress_value = prm->stress_value;
    e->prm.calculate_strain = prm->calculate_strain;
    e->prm.solver = prm->solver;
    e->prm.solver_tol = prm->solver_tol;
    e->prm.max_iters = prm->max_iters;
    e->prm.precond_theta = prm->precond_theta;
    e->prm.neumann_theta = prm->neumann_theta;
    e->prm.gmres_restart = prm->gmres_restart < 2 ? restart_alloc : std::min(prm->gmres_restart, restart_alloc);
    e->restart = e->prm.gmres_restart;
    e->prec = prm->prec;
    e->cutoff_multiplier = prm->cutoff_multiplier;
    e->update_cutoff();
    const int ncell = e->G * e->G;
    if (ncell > e->ncell_alloc) {
        int **arrs[] = {&e->d_cell_count, &e->d_cell_start, &e->d_cell_fill};
        for (int **a : arrs) {
            cudaFree(*a);
            *a = nullptr;
            if (cudaMalloc(a, sizeof(int) * (ncell + 1)) != cudaSuccess) return fail(SDDDST_ERR_NOMEM, "cell arrays");
        }
        e->ncell_alloc = ncell;
    }
    return SDDDST_OK;
}

int sdddst_solve_csc(void *ctx, const int *Ap, const int *Ai, const double *Ax, const double *b, double *x,
                     int *iterations)
{
    if (!ctx || !Ap || !Ai || !Ax || !b || !x) return fail(SDDDST_ERR_INVALID, "null argument");
    sd::Engine *e = E(ctx);
    e->pre_assembled = false; // the stored pattern no longer matches the next attempt
    cudaSetDevice(e->device);
    const int n = e->n;
    sd::learned_invalidate(*e); // the CSR is replaced below
    try {
        // CSC of A -> CSR rows of G = A - I with the diagonal in each row's first slot
        std::vector<int> cnt(n + 1, 1);
        for (int j = 0; j < n; ++j)
            for (int q = Ap[j]; q < Ap[j + 1]; ++q) {
                int i = Ai[q];
                if (i < 0 || i >= n) return fail(SDDDST_ERR_INVALID, "row index out of range");
                if (i != j) cnt[i]++;
            }
        std::vector<int> rp(n + 1, 0);
        for (int i = 0; i < n; ++i) rp[i + 1] = rp[i] + cnt[i];
        const long nnz = rp[n];
        std::vector<int> cl(nnz), fill(n);
        std::vector<double> vl(nnz, 0.0), gd(n, -1.0), ones(n, 1.0);
        for (int i = 0; i < n; ++i) {
            fill[i] = rp[i] + 1;
            cl[rp[i]] = i;
        }
        for (int j = 0; j < n; ++j)
            for (int q = Ap[j]; q < Ap[j + 1]; ++q) {
                int i = Ai[q];
                if (i == j) gd[i] += Ax[q];
                else {
                    cl[fill[i]] = j;
                    vl[fill[i]++] = Ax[q];
                }
            }
        for (int i = 0; i < n; ++i) vl[rp[i]] = gd[i];
        if (nnz > e->nnz_cap) {
            if (sd::alloc_csr_values(*e, nnz + nnz / 4)) return fail(SDDDST_ERR_NOMEM, "CSR allocation");
            e->nnz_cap = nnz + nnz / 4;
        }
        e->nnz = nnz;
        e->col_s_valid = false; // a caller's matrix: no cell-sorted column positions
        e->col_s16_valid = false;
        cudaMemcpyAsync(e->d_rowptr, rp.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice, e->st);
        cudaMemcpyAsync(e->d_col, cl.data(), sizeof(int) * nnz, cudaMemcpyHostToDevice, e->st);
        std::vector<float> vf;
        if (e->valf) {
            vf.assign(vl.begin(), vl.end());
            cudaMemcpyAsync(e->d_valf, vf.data(), sizeof(float) * nnz, cudaMemcpyHostToDevice, e->st);
        } else {
            cudaMemcpyAsync(e->d_val, vl.data(), sizeof(double) * nnz, cudaMemcpyHostToDevice, e->st);
        }
        cudaMemcpyAsync(e->d_gdiag, gd.data(), sizeof(double) * n, cudaMemcpyHostToDevice, e->st);
        cudaMemcpyAsync(e->d_dvec, ones.data(), sizeof(double) * n, cudaMemcpyHostToDevice, e->st);
        cudaMemcpyAsync(e->d_g, b, sizeof(double) * n, cudaMemcpyHostToDevice, e->st);
        if (int rc = e->sync_check("solve_csc upload")) return from_engine(e, rc);
        // J(h=1, d=1) = I + (1+1)/2 * 1 * (A - I) = A
        if (int rc = e->prepare_solver(1.0)) return from_engine(e, rc);
        int rc = e->solve(1.0, e->d_g, e->d_sol);
        if (iterations) *iterations = e->last_iters;
        if (rc) return from_engine(e, rc);
        cudaMemcpyAsync(x, e->d_sol, sizeof(double) * n, cudaMemcpyDeviceToHost, e->st);
        return from_engine(e, e->sync_check("solve_csc"));
    } catch (const std::exception &ex) {
        return fail(SDDDST_ERR_NOMEM, ex.what());
    }
}

int sdddst_jacobian(void *ctx, double h, const double *xyb, int *row_ptr, int *col, double *val, double *dvec,
                    long cap, long *nnz)
{
    if (!ctx || !xyb || !row_ptr || !nnz) return fail(SDDDST_ERR_INVALID, "null argument");
    sd::Engine *e = E(ctx);
    if (int rc = check_finite(xyb, 3L * e->n, "configuration")) return rc;
    cudaSetDevice(e->device);
    try {
        ScratchConfig sc(e, xyb);
        if (int rc = e->assemble(e->d_xs)) return from_engine(e, rc);
        *nnz = e->nnz;
        if (e->nnz > cap || !col || !val || !dvec) return fail(SDDDST_ERR_CAPACITY, "output capacity too small");
        sd::launch_make_dvec(*e, h, e->d_dvec, e->st);
        double *tmp = nullptr;
        if (cudaMalloc(&tmp, sizeof(double) * e->nnz) != cudaSuccess) return fail(SDDDST_ERR_NOMEM, "export buffer");
        sd::launch_export_jacobian(*e, h, e->d_dvec, tmp, e->st);
        cudaMemcpyAsync(row_ptr, e->d_rowptr, sizeof(int) * (e->n + 1), cudaMemcpyDeviceToHost, e->st);
        cudaMemcpyAsync(col, e->d_col, sizeof(int) * e->nnz, cudaMemcpyDeviceToHost, e->st);
        cudaMemcpyAsync(val, tmp, sizeof(double) * e->nnz, cudaMemcpyDeviceToHost, e->st);
        cudaMemcpyAsync(dvec, e->d_dvec, sizeof(double) * e->n, cudaMemcpyDeviceToHost, e->st);
        int rc = e->sync_check("jacobian export");
        cudaFree(tmp);
        return from_engine(e, rc);
    } catch (const std::exception &ex) {
        return fail(SDDDST_ERR_NOMEM, ex.what());
    }
}

int sdddst_solve(void *ctx, double h, const double *xyb, const double *rhs, double *x, int *iterations)
{
    if (!ctx || !xyb || !rhs || !x) return fail(SDDDST_ERR_INVALID, "null argument");
    sd::Engine *e = E(ctx);
    if (int rc = check_finite(xyb, 3L * e->n, "configuration")) return rc;
    cudaSetDevice(e->device);
    try {
        ScratchConfig sc(e, xyb);
        if (int rc = e->assemble(e->d_xs)) return from_engine(e, rc);
        sd::launch_make_dvec(*e, h, e->d_dvec, e->st);
        if (int rc = e->prepare_solver(h)) return from_engine(e, rc);
        cudaMemcpyAsync(e->d_g, rhs, sizeof(double) * e->n, cudaMemcpyHostToDevice, e->st);
        int rc = e->solve(h, e->d_g, e->d_sol);
        if (iterations) *iterations = e->last_iters;
        if (rc) return from_engine(e, rc);
        cudaMemcpyAsync(x, e->d_sol, sizeof(double) * e->n, cudaMemcpyDeviceToHost, e->st);
        return from_engine(e, e->sync_check("solve"));
    } catch (const std::exception &ex) {
        return fail(SDDDST_ERR_NOMEM, ex.what());
    }
}

int sdddst_step(void *ctx, int *accepted)
{
    if (!ctx) return fail(SDDDST_ERR_INVALID, "null argument");
    sd::Engine *e = E(ctx);
    cudaSetDevice(e->device);
    try {
        return from_engine(e, e->step(accepted));
    } catch (const std::exception &ex) {
        return fail(SDDDST_ERR_NOMEM, ex.what());
    }
}

int sdddst_run(void *ctx, int accepted_target, int max_attempts, int *accepted, int *attempts)
{
    if (!ctx) return fail(SDDDST_ERR_INVALID, "null argument");
    int acc = 0, att = 0;
    while (acc < accepted_target && att < max_attempts) {
        int a = 0;
        int rc = sdddst_step(ctx, &a);
        att++;
        if (rc) {
            if (accepted) *accepted = acc;
            if (attempts) *attempts = att;
            return rc;
        }
        acc += a;
    }
    if (accepted) *accepted = acc;
    if (attempts) *attempts = att;
    return SDDDST_OK;
}

int sdddst_state_device(void *ctx, double **x, double **y, double **b)
{
    if (!ctx) return fail(SDDDST_ERR_INVALID, "null argument");
    sd::Engine *e = E(ctx);
    if (x) *x = e->d_x0;
    if (y) *y = e->d_y;
    if (b) *b = e->d_b;
    return SDDDST_OK;
}

int sdddst_upload_positions(void *ctx, const double *x, int recompute)
{
    if (!ctx || !x) return fail(SDDDST_ERR_INVALID, "null argument");
    sd::Engine *e = E(ctx);
    if (int rc = check_finite(x, e->n, "positions")) return rc;
    cudaSetDevice(e->device);
    // staged and compared: a round trip of the held state keeps the next
    // attempt's stage I assembly; any changed position drops it
    cudaMemcpyAsync(e->d_xs, x, sizeof(double) * e->n, cudaMemcpyHostToDevice, e->st);
    cudaMemsetAsync(e->d_flag, 0, sizeof(int), e->st);
    copy_compare_kernel<<<(e->n + 255) / 256, 256, 0, e->st>>>(e->n, e->d_xs, e->d_x0, e->d_flag);
    int changed = 1;
    cudaMemcpyAsync(&changed, e->d_flag, sizeof(int), cudaMemcpyDeviceToHost, e->st);
    if (int rc = e->sync_check("upload positions")) return from_engine(e, rc);
    if (changed || recompute) e->pre_assembled = false;
    if (recompute) {
        e->cur_stress = SDDDST_STAGE_ORIGINAL;
        e->stress_calc(e->sim_time, SDDDST_STAGE_ORIGINAL, e->strain);
        e->speeds(e->d_x0, e->d_v0, e->d_S0, SDDDST_STAGE_ORIGINAL, false);
    }
    return from_engine(e, e->sync_check("upload positions"));
}

int sdddst_download_positions(void *ctx, double *x)
{
    if (!ctx || !x) return fail(SDDDST_ERR_INVALID, "null argument");
    sd::Engine *e = E(ctx);
    cudaSetDevice(e->device);
    cudaMemcpyAsync(x, e->d_x0, sizeof(double) * e->n, cudaMemcpyDeviceToHost, e->st);
    return from_engine(e, e->sync_check("download positions"));
}

int sdddst_stream(void *ctx, void **stream)
{
    if (!ctx || !stream) return fail(SDDDST_ERR_INVALID, "null argument");
    *stream = (void *)E(ctx)->st;
    return SDDDST_OK;
}

int sdddst_profile_pair_sum(void *ctx, int reps, double *ms_per_launch)
{
    if (!ctx || !ms_per_launch || reps < 1) return fail(SDDDST_ERR_INVALID, "bad argument");
    sd::Engine *e = E(ctx);
    cudaSetDevice(e->device);
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    sd::launch_pair_sum(*e, e->d_x0, e->st, e->prm.pairsum, 0.0); // warm-up
    cudaEventRecord(a, e->st);
    for (int r = 0; r < reps; ++r) sd::launch_pair_sum(*e, e->d_x0, e->st, e->prm.pairsum, 0.0);
    cudaEventRecord(b, e->st);
    int rc = e->sync_check("profile pair sum");
    float ms = 0.f;
    if (!rc) cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    e->launches += (e->prm.pairsum == SDDDST_PAIRSUM_FP32 ? 3 : 2) * (reps + 1);
    *ms_per_launch = ms / reps;
    return from_engine(e, rc);
}

// Internal counters of the learned correction (not part of the public
// header): network inferences, rescales onto a second step size of the same
// assembly, and remaps onto a new assembly.
int sdddst_internal_learned_counts(void *ctx, long *inferences, long *rescales, long *remaps)
{
    if (!ctx || !inferences || !rescales || !remaps) return fail(SDDDST_ERR_INVALID, "null argument");
    sd::learned_counts(*E(ctx), inferences, rescales, remaps);
    return SDDDST_OK;
}

// Internal check of the exclusive scan the assembly and the preconditioner
// build use (not part of the public header): out[0..m] from in[0..m-1], both
// device pointers, on the context's stream, with scratch sized for m.
int sdddst_internal_scan(void *ctx, const int *in, int m, int *out)
{
    if (!ctx || !in || !out || m < 1) return fail(SDDDST_ERR_INVALID, "bad argument");
    sd::Engine *e = E(ctx);
    cudaSetDevice(e->device);
    int *saved = e->d_scan_tmp;
    const int saved_cap = e->scan_tmp_cap;
    const int need = 2 * ((m + 2047) / 2048) + 2;
    int *tmp = nullptr;
    if (need > saved_cap) {
        if (cudaMalloc(&tmp, sizeof(int) * need) != cudaSuccess) return fail(SDDDST_ERR_NOMEM, "scan scratch");
        e->d_scan_tmp = tmp;
        e->scan_tmp_cap = need;
    }
    e->launches += sd::launch_scan(*e, in, m, out, e->st);
    const int rc = e->sync_check("scan");
    e->d_scan_tmp = saved;
    e->scan_tmp_cap = saved_cap;
    if (tmp) cudaFree(tmp);
    return from_engine(e, rc);
}

int sdddst_profile_direct(void *ctx, double h, int reps, double *factor_ms, double *solve_ms)
{
    if (!ctx || !factor_ms || !solve_ms || reps < 1 || !(h > 0)) return fail(SDDDST_ERR_INVALID, "bad argument");
    sd::Engine *e = E(ctx);
    if (e->prm.solver != SDDDST_SOLVER_DIRECT && e->prm.solver != SDDDST_SOLVER_DIRECT_MIXED)
        return fail(SDDDST_ERR_INVALID, "the context's solver is not the sparse LU");
    cudaSetDevice(e->device);
    try {
        if (int rc = e->assemble(e->d_x0)) return from_engine(e, rc);
        sd::launch_make_dvec(*e, h, e->d_dvec, e->st);
        if (int rc = sd::direct_factor(*e, h, e->d_dvec)) return from_engine(e, rc); // warm-up
        cudaEvent_t a, b, c;
        cudaEventCreate(&a);
        cudaEventCreate(&b);
        cudaEventCreate(&c);
        cudaEventRecord(a, e->st);
        int rc = 0;
        for (int r = 0; r < reps && !rc; ++r) rc = sd::direct_factor(*e, h, e->d_dvec);
        cudaEventRecord(b, e->st);
        for (int r = 0; r < reps && !rc; ++r) rc = sd::direct_apply(*e, e->d_v0, e->d_sol);
        cudaEventRecord(c, e->st);
        if (!rc) rc = e->sync_check("profile direct");
        float m1 = 0.f, m2 = 0.f;
        if (!rc) {
            cudaEventElapsedTime(&m1, a, b);
            cudaEventElapsedTime(&m2, b, c);
        }
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        cudaEventDestroy(c);
        *factor_ms = m1 / reps;
        *solve_ms = m2 / reps;
        return from_engine(e, rc);
    } catch (const std::exception &ex) {
        return fail(SDDDST_ERR_NOMEM, ex.what());
    }
}

int sdddst_precond_apply(void *ctx, double h, int k, const double *in_device, double *out_device,
                         int *block_of_device)
{
    if (!ctx || !in_device || !out_device || k < 1 || !(h > 0)) return fail(SDDDST_ERR_INVALID, "bad argument");
    sd::Engine *e = E(ctx);
    cudaSetDevice(e->device);
    try {
        if (int rc = e->assemble(e->d_x0)) return from_engine(e, rc);
        sd::launch_make_dvec(*e, h, e->d_dvec, e->st);
        if (int rc = sd::precond_build(*e, h, e->d_dvec)) return from_engine(e, rc);
        for (int q = 0; q < k; ++q) sd::precond_apply(*e, in_device + (size_t)q * e->n, out_device + (size_t)q * e->n);
        if (block_of_device)
            cudaMemcpyAsync(block_of_device, e->pc.blk_of, sizeof(int) * e->n, cudaMemcpyDeviceToDevice, e->st);
        return from_engine(e, e->sync_check("precond apply"));
    } catch (const std::exception &ex) {
        return fail(SDDDST_ERR_NOMEM, ex.what());
    }
}

int sdddst_set_preconditioner_weights(void *ctx, const unsigned short *bf16, long count)
{
    if (!ctx || !bf16) return fail(SDDDST_ERR_INVALID, "null argument");
    sd::Engine *e = E(ctx);
    cudaSetDevice(e->device);
    return from_engine(e, sd::learned_set_weights(*e, bf16, count));
}

int sdddst_learned_train_init(void *ctx, const float *weights, long count)
{
    if (!ctx || !weights) return fail(SDDDST_ERR_INVALID, "null argument");
    if (int rc = check_finite_f(weights, count, "weights")) return rc;
    sd::Engine *e = E(ctx);
    cudaSetDevice(e->device);
    return from_engine(e, sd::learned_train_init(*e, weights, count));
}

int sdddst_learned_train_step(void *ctx, double h, int probes, double lr, unsigned long long seed, int apply,
                              double *loss2, float *grad)
{
    if (!ctx || !(h > 0) || !(lr >= 0)) return fail(SDDDST_ERR_INVALID, "bad argument");
    sd::Engine *e = E(ctx);
    cudaSetDevice(e->device);
    try {
        return from_engine(e, sd::learned_train_step(*e, h, probes, lr, seed, apply != 0, loss2, grad));
    } catch (const std::exception &ex) {
        return fail(SDDDST_ERR_NOMEM, ex.what());
    }
}

int sdddst_learned_train_weights(void *ctx, float *weights, long count)
{
    if (!ctx || !weights) return fail(SDDDST_ERR_INVALID, "null argument");
    sd::Engine *e = E(ctx);
    cudaSetDevice(e->device);
    return from_engine(e, sd::learned_train_weights(*e, weights, count));
}

int sdddst_learned_correction(void *ctx, double h, float *values, long cap, long *nnz)
{
    if (!ctx || !values || !nnz || !(h > 0)) return fail(SDDDST_ERR_INVALID, "bad argument");
    sd::Engine *e = E(ctx);
    cudaSetDevice(e->device);
    try {
        if (!e->learned) return fail(SDDDST_ERR_INVALID, "no learned preconditioner weights loaded");
        if (!e->d_xasm && cudaMalloc(&e->d_xasm, sizeof(double) * e->n) != cudaSuccess)
            return fail(SDDDST_ERR_NOMEM, "positions buffer");
        if (int rc = e->assemble(e->d_x0)) return from_engine(e, rc);
        cudaMemcpyAsync(e->d_xasm, e->d_x0, sizeof(double) * e->n, cudaMemcpyDeviceToDevice, e->st);
        sd::launch_make_dvec(*e, h, e->d_dvec, e->st);
        if (int rc = sd::precond_build(*e, h, e->d_dvec)) return from_engine(e, rc);
        if (int rc = sd::learned_build(*e, h, e->d_dvec, e->d_xasm, false)) return from_engine(e, rc);
        *nnz = e->nnz;
        return from_engine(e, sd::learned_export(*e, values, cap));
    } catch (const std::exception &ex) {
        return fail(SDDDST_ERR_NOMEM, ex.what());
    }
}

int sdddst_solver_stats(void *ctx, long *solves, long *iterations)
{
    if (!ctx) return fail(SDDDST_ERR_INVALID, "null argument");
    if (solves) *solves = E(ctx)->solves;
    if (iterations) *iterations = E(ctx)->iterations;
    return SDDDST_OK;
}

int sdddst_solver_recoveries(void *ctx, long *rebuilds, long *fallbacks, long *redone)
{
    if (!ctx) return fail(SDDDST_ERR_INVALID, "null argument");
    if (rebuilds) *rebuilds = E(ctx)->stalls;
    if (fallbacks) *fallbacks = E(ctx)->fallbacks;
    if (redone) *redone = E(ctx)->redone;
    return SDDDST_OK;
}

int sdddst_ev_hessian(void *ctx, const double *xyb, double *H)
{
    if (!ctx || !xyb || !H) return fail(SDDDST_ERR_INVALID, "null argument");
    sd::Engine *e = E(ctx);
    if (int rc = check_finite(xyb, 3L * e->n, "configuration")) return rc;
    cudaSetDevice(e->device);
    try {
        ScratchConfig sc(e, xyb);
        if (int rc = sd::ev_hessian(*e, e->d_xs)) return from_engine(e, rc);
        cudaMemcpyAsync(H, sd::ev_hessian_ptr(*e), sizeof(double) * (size_t)e->n * e->n, cudaMemcpyDeviceToHost,
                        e->st);
        return from_engine(e, e->sync_check("Hessian"));
    } catch (const std::exception &ex) {
        return fail(SDDDST_ERR_NOMEM, ex.what());
    }
}

int sdddst_ev_analyze(void *ctx, const double *xyb, double sim_time, double *eigenvalues, double *participation,
                      double *burgers_sum, double *gan, double *speeds, double *eigenvectors, int nvec,
                      double *derivatives, double *correlations, int corr_bins)
{
    if (!ctx || !xyb || nvec < 0 || corr_bins < 0 || (correlations && corr_bins == 0) ||
        (nvec > 0 && !eigenvectors))
        return fail(SDDDST_ERR_INVALID, "bad argument");
    sd::Engine *e = E(ctx);
    if (int rc = check_finite(xyb, 3L * e->n, "configuration")) return rc;
    if (!(corr_bins <= 4096)) return fail(SDDDST_ERR_INVALID, "correlation sampling size above 4096");
    cudaSetDevice(e->device);
    try {
        ScratchConfig sc(e, xyb);
        const int n = e->n;
        // TimeSeriesProcessor::run: the stress at the configuration's time
        // (Original), then calculateSpeeds without precision-handler updates
        e->stress_calc(sim_time, 0, e->strain);
        e->speeds(e->d_xs, e->d_Stmp, e->d_w, 0, false);
        const bool deriv = derivatives && e->prm.stress_kind == SDDDST_STRESS_FIXED_RATE;
        if (int rc = sd::ev_analyze(*e, e->d_xs, e->d_Stmp, deriv, e->prm.stress_rate, correlations ? corr_bins : 0))
            return from_engine(e, rc);
        const size_t nb = sizeof(double) * n;
        const double *obs = sd::ev_observables(*e);
        if (eigenvalues) cudaMemcpyAsync(eigenvalues, sd::ev_values(*e), nb, cudaMemcpyDeviceToHost, e->st);
        if (participation) cudaMemcpyAsync(participation, obs, nb, cudaMemcpyDeviceToHost, e->st);
        if (burgers_sum) cudaMemcpyAsync(burgers_sum, obs + n, nb, cudaMemcpyDeviceToHost, e->st);
        if (gan) cudaMemcpyAsync(gan, obs + 2 * (size_t)n, nb, cudaMemcpyDeviceToHost, e->st);
        if (derivatives) cudaMemcpyAsync(derivatives, obs + 3 * (size_t)n, nb, cudaMemcpyDeviceToHost, e->st);
        if (speeds) cudaMemcpyAsync(speeds, e->d_Stmp, nb, cudaMemcpyDeviceToHost, e->st);
        const int nv = std::min(nvec, n);
        if (nv > 0) cudaMemcpyAsync(eigenvectors, sd::ev_vectors(*e), nb * nv, cudaMemcpyDeviceToHost, e->st);
        if (correlations)
            cudaMemcpyAsync(correlations, sd::ev_correlations(*e), nb * 3 * (size_t)corr_bins * corr_bins,
                            cudaMemcpyDeviceToHost, e->st);
        return from_engine(e, e->sync_check("eigenvalue analysis"));
    } catch (const std::exception &ex) {
        return fail(SDDDST_ERR_NOMEM, ex.what());
    }
}

int sdddst_ev_timings(void *ctx, double *ms5)
{
    if (!ctx || !ms5) return fail(SDDDST_ERR_INVALID, "null argument");
    sd::ev_timings(*E(ctx), ms5);
    return SDDDST_OK;
}

int sdddst_direct_stats(void *ctx, long *factorizations, long *perturbed, double *flops, long *front_doubles,
                        int *fronts, int *depth)
{
    if (!ctx) return fail(SDDDST_ERR_INVALID, "null argument");
    long f = 0, p = 0, fd = 0;
    double fl = 0.0;
    int nf = 0, dp = 0;
    sd::direct_stats(*E(ctx), &f, &p, &fl, &fd, &nf, &dp);
    if (factorizations) *factorizations = f;
    if (perturbed) *perturbed = p;
    if (flops) *flops = fl;
    if (front_doubles) *front_doubles = fd;
    if (fronts) *fronts = nf;
    if (depth) *depth = dp;
    return SDDDST_OK;
}

long sdddst_kernel_launches(void *ctx) { return ctx ? E(ctx)->launches : 0; }

} // extern "C"
