// Host-side engine of one simulated system: device buffers, parameters and
// the step driver.  Mirrors the state of the reference's SimulationData +
// Simulation + PrecisionHandler (include/simulation_data.h:69-144,
// include/simulation.h:73-85, include/precision_handler.h:54-59) with the
// vectors resident in HBM as structure-of-arrays doubles.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/sdddst_b200.h"

namespace sd {

// One cluster block-Jacobi preconditioner: the block structure of J(h) and
// the blocks' inverses (precond.cu).
struct Cluster {
    int *ptr = nullptr, *parent = nullptr, *tmp = nullptr, *tmp2 = nullptr, *members = nullptr;
    int *blk_of = nullptr, *loc = nullptr, *count = nullptr, *fill = nullptr, *start = nullptr;
    int *nblk = nullptr, *bbase = nullptr, *bstart = nullptr, *blen = nullptr, *sq = nullptr;
    int *off = nullptr;
    int *flag = nullptr; // set by the inversion when a block is singular
    double *binv = nullptr;
    long binv_cap = 0;
};

struct Engine {
    // ---- sizes and parameters
    int n = 0, p = 0, device = 0;
    sdddst_params prm{};
    double cutoff_multiplier = 1.0, cutoff = 1.0, cutoff_sqr = 1.0, one_per_cutoff_sqr = 1.0;
    double prec = 1e-8, A = 0, KASQR = 0;
    int ic = 2;
    cudaStream_t st = nullptr;

    // ---- configuration and step vectors (N doubles each)
    double *d_x0 = nullptr, *d_y = nullptr, *d_b = nullptr; // accepted configuration
    double *d_xb = nullptr, *d_x1 = nullptr, *d_x2 = nullptr, *d_xs = nullptr;
    double *d_v0 = nullptr, *d_v0b = nullptr, *d_vs = nullptr, *d_vs2 = nullptr;
    double *d_S0 = nullptr, *d_S1 = nullptr, *d_Stmp = nullptr; // pair+defect sums without tau_ext
    double *d_g = nullptr, *d_sol = nullptr, *d_dvec = nullptr;
    double *d_tol = nullptr, *d_tol_last = nullptr;
    unsigned long long *d_minr2 = nullptr;
    double *d_part = nullptr;
    double *d_pdx = nullptr, *d_pdy = nullptr;
    double *d_ys = nullptr, *d_bs = nullptr; // scratch y, b of caller-supplied configurations
    double *d_xw = nullptr;                  // positions wrapped into [-0.5, 0.5) (mixed pair sum)
    double *d_tab_xy = nullptr, *d_tab_dx = nullptr; // tabulated field: remainder tables (null: analytic)
    double *d_minr2_out = nullptr;           // optional per-dislocation min distance output

    // ---- cell list of the cutoff-neighbour search
    int G = 1; // cells per axis
    int ncell_alloc = 0; // cell arrays hold ncell_alloc + 1 entries
    int *d_cell = nullptr, *d_cell_count = nullptr, *d_cell_start = nullptr, *d_cell_fill = nullptr;
    int *d_sorted = nullptr;

    // ---- CSR of the unit-step Jacobian part G = H / h (diagonal in slot 0 of each row)
    int *d_rowcnt = nullptr, *d_rowptr = nullptr, *d_col = nullptr;
    double *d_val = nullptr;   // FP64 values (plain path)
    float *d_valf = nullptr;   // FP32 values (mixed path)
    bool valf = false;         // which of the two holds G
    double *d_gdiag = nullptr; // G_ii in FP64 (both paths)
    int *d_col_s = nullptr;    // column positions in the cell-sorted order (SpMV gathers; diagonal slot unused)
    double *d_vsort = nullptr; // SpMV input gathered into the cell-sorted order
    double *d_xsrt = nullptr, *d_ysrt = nullptr, *d_bsrt = nullptr; // x, y, b in the cell-sorted order
    bool col_s_valid = false;  // d_col_s matches the assembled CSR
    unsigned short *d_col_s16 = nullptr; // d_col_s in 16 bits (systems of at most 65536), the SpMV's copy
    bool col_s16_valid = false;
    int *d_scan_tmp = nullptr; // chunk totals and offsets of launch_scan
    int scan_tmp_cap = 0;
    const int *spmv_sorted = nullptr; // the sorted list d_col_s refers to
    double *d_hrow = nullptr;  // per-row step size of a batch of systems (null: one system, scalar h)
    long nnz_cap = 0, nnz = 0;
    int *d_flag = nullptr; // device-side error flag of the assembly
    bool assembled_valid = false;
    const double *assembled_for = nullptr;

    // ---- Krylov workspace
    int restart = 30;
    double *d_V = nullptr, *d_w = nullptr, *d_z = nullptr, *d_r = nullptr, *d_hcol = nullptr;
    double *d_partials = nullptr, *d_scal = nullptr, *d_y_small = nullptr;
    int red_blocks = 0, gs_blocks = 0;
    double *h_scal = nullptr; // pinned
    int last_iters = 0;
    double last_resid = 0.0;
    long solves = 0, iterations = 0;      // solver statistics
    long stalls = 0;                      // solves repeated with a rebuilt preconditioner
    long fallbacks = 0;                   // stalled learned-preconditioned solves redone by the sparse LU
    double *d_hrec = nullptr;             // per-iteration Gram-Schmidt records
    double *h_hrec = nullptr;             // pinned copy
    unsigned int *d_counter = nullptr;    // last-block ticket of the fused reductions
    bool coop_gs = false;                 // one cooperative launch per Gram-Schmidt step
    int gmres_hint = 4;                   // iterations of the last solve (first convergence check)
    double *d_gs_partials = nullptr;      // its per-CTA partial sums (3 x gs_blocks x 32)
    // device-resident GMRES (fused_gmres.cu): partial sums, per-system status,
    // and the second system's Krylov basis and vectors (joint stage I + II)
    double *d_fpart = nullptr, *d_fstatus = nullptr, *h_fstatus = nullptr;
    int *d_fctr = nullptr; // row counters of the device-resident GMRES's SpMV passes
    int2 *d_fsrow = nullptr; // per cell-sorted position: its CSR row's (start, end)
    double *d_V2 = nullptr, *d_w2 = nullptr, *d_z2 = nullptr, *d_zs2 = nullptr;
    double *d_gI = nullptr, *d_solI = nullptr, *d_dvecI = nullptr, *d_vsI = nullptr; // stage I's g, solution, d, speed
    bool fused = false;                   // the cluster solver runs device-resident (set at init)
    // optimistic attempts (no host round trip until the stages end): the
    // statuses they leave on the device, read back in one copy, and the
    // tolerance snapshot restored when an attempt has to be redone
    int *d_astat = nullptr;               // per deferred assembly: entry total, fill flag
    double *d_tol_snap = nullptr;
    double *h_status = nullptr;           // pinned: fused statuses, assembly and preconditioner checks, scalars
    long redone = 0;                      // attempts redone with waits after a deferred failure
    // side stream of the optimistic attempts: assemblies and preconditioner
    // builds beside the pair sum at the same configuration
    cudaStream_t st2 = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    bool pre_assembled = false;           // the CSR holds the next attempt's stage I assembly (at x0)

    // ---- cluster block-Jacobi preconditioners (precond.cu): pc for the
    // solves of the engine's generic path and of stage II/III, pc2 for stage
    // I's J(h) while the joint stage I + II solve holds both
    Cluster pc, pc2;

    // ---- sparse LU (direct.cu)
    void *direct = nullptr;

    // ---- learned preconditioner correction (learned.cu)
    void *learned = nullptr;
    double *d_xasm = nullptr; // positions of the last assembly (learned features, LU fallback)

    // ---- eigenvalue analysis (ev.cu): dense Hessian, eigenpairs, observables
    void *ev = nullptr;

    // ---- host scalars (SimulationData / Simulation members)
    double step_size = 1.0, sim_time = 0.0, strain = 0.0;
    double energy = 0.0, energy_accum = 0.0, vsquare = 0.0, vsquare1 = 0.0, vsquare2 = 0.0;
    double sum_avg_speed = 0.0, last_ratio = 0.0;
    double stress_vals[4] = {0, 0, 0, 0};
    long succ = 0, failed = 0;
    bool first_step = true, init_speed_needed = true, successful_step = true;
    int cur_stress = 0;

    long launches = 0;
    std::string err;
    bool batch_backend = false; // buffers for a batch of systems (batch.cu allocates its own pair-sum slabs)

    ~Engine();
    int init(const sdddst_params &prm, const double *xyb, const double *pd);
    void update_cutoff();

    // reference operations
    int speeds(const double *x, double *v_out, double *S_out, int stress_type, bool update_tol);
    int assemble(const double *x);
    int solve(double h, const double *rhs, double *x_out);
    // per matrix: preconditioner set-up; same_assembly: the matrix shares the
    // previous set-up's assembly (only h differs)
    int prepare_solver(double h, bool same_assembly = false);
    int integrate(double h, double *xn, const double *xo, bool use2, bool init_speed, int origin, int end,
                  bool reuse_assembly);
    // calculateG of one chord-Newton iteration of one stage: speeds at the
    // iterate (csp) or the initial speeds, then g (simulation.cpp:133-193)
    int stage_residual(double h, int it, double *xn, const double *xo, bool use2, bool init_speed, int origin,
                       int end, double *csp0, const double *dvec, double *g);
    // stage I (h) and stage II (h/2) from the accepted configuration with
    // their solves in one device-resident launch per Newton iteration
    int stages_one_two();
    int stages_sync(double *ratio);
    int stages_async(double *ratio, bool *ok);
    int finish_step(double ratio, int *accepted);
    int abs_and_sq(const double *v, double *sum_abs, double *sum_sq);
    // the calculateSpeeds of a stage's initial configuration (calculateG's
    // first part, simulation.cpp:143-160)
    int init_speeds(int origin, const double *xo, bool use2);
    int side_streams();                   // creates st2 and its events once
    void fork_side();                     // st2 waits for st; launches go to st2 until join_side
    void end_side();                      // launches back on st; the side work is recorded
    void join_side();                     // st waits for the recorded side work
    int solve_fused(double h, const double *dvec, Cluster &c, const double *rhs, double *x);
    int step(int *accepted);
    int set_state_host(const double *xyb, double step, double t, double e, double strain, int first);

    // stress protocol (host scalars)
    void stress_calc(double t, int type, double strain_now);
    double stress_get(int type) const;
    bool zero_stress() const { return prm.stress_kind == SDDDST_STRESS_ZERO; }

    // device reductions (results on host)
    int sum_sq(const double *v, double *out);
    int sum_abs(const double *v, double *out);
    int strain_inc(const double *xo, const double *xn, double *out);
    int max_ratio(double *out);
    int stage_scalars(double *vs1, double *vs2, double *ratio);
    int sync_check(const char *what);
};

// ---- launchers (one .cu file each)
int pair_tile_size(int n);
size_t pair_part_doubles(int n);
void launch_pair_sum(const Engine &e, const double *x, cudaStream_t st, int mode, double r2_track);
void launch_speeds_finish(const Engine &e, const double *x, double tau_ext, double *S, double *v, int update_tol,
                          cudaStream_t st);
void launch_add_stress(const Engine &e, const double *S, double tau_ext, double *v, cudaStream_t st);
void launch_speeds_raw(int n, const double *x, const double *y, const double *b, double tau_ext, double *part,
                       double *v, cudaStream_t st);

int jacobian_assemble(Engine &e, const double *x, bool defer = false);
void launch_csr_guard(Engine &e, int *stat);
int tabulated_build(Engine &e);
int alloc_csr_values(Engine &e, long cap);
// Exclusive scan of m ints (out[0] = 0, out[k+1] = sum_{<=k}); returns the
// number of kernels launched.
int launch_scan(Engine &e, const int *in, int m, int *out, cudaStream_t st);
// Coupling threshold of the cluster preconditioner: the caller's setting, else
// 0.01 for the cluster-preconditioned GMRES (fewest step-time on the N=32768
// workload: 0.01, 0.02, 0.05, 0.1, 0.2 give 11.20, 11.27, 11.59, 11.92,
// 12.30 ms per attempt) and 0.05 under the learned and analytic corrections
// (the network was trained on blocks built at 0.05).
double cluster_theta(const Engine &e);
void launch_make_dvec(const Engine &e, double h, double *dvec, cudaStream_t st);
void launch_export_jacobian(const Engine &e, double h, const double *dvec, double *val_out, cudaStream_t st);

void launch_spmv_J(Engine &e, double h, const double *dvec, const double *v, double *y, cudaStream_t st);
int gmres_solve(Engine &e, double h, const double *dvec, const double *rhs, double *x, int precond);
bool gs_coop_supported(int device, int blocks);

constexpr int kAttemptSlots = 8; // solve statuses of one optimistic attempt (2 ic joint + ic stage III)
// |v0|^2, |v0b|^2 and the error ratio of the attempt into d_scal[0..2] (no wait)
void launch_stage_scalars(Engine &e);
void launch_fill(Engine &e, double *p, double v);
void launch_residual_g(const Engine &e, double h, const double *xn, const double *xo, const double *csp,
                       const double *isp, const double *dvec, double *g, cudaStream_t st);
void launch_axpy_update(const Engine &e, double *xn, const double *sol, cudaStream_t st);

int reduce_sum(Engine &e, const double *a, const double *b, int n, int op, double *out);
void set_last_error(const std::string &msg);

int precond_alloc(Engine &e, Cluster &c);
void precond_free(Cluster &c);
// Builds c for J(h); with check, waits for the build and verifies the block
// count and the inversions (else the caller checks later with precond_check).
int precond_build(Engine &e, Cluster &c, double h, const double *dvec, bool check = true);
int precond_check(Engine &e, const Cluster &c);
inline int precond_build(Engine &e, double h, const double *dvec) { return precond_build(e, e.pc, h, dvec); }
void precond_apply(Engine &e, const Cluster &c, const double *v, double *z);
inline void precond_apply(Engine &e, const double *v, double *z) { precond_apply(e, e.pc, v, z); }

int direct_analyse(Engine &e, const double *x);
int direct_factor(Engine &e, double h, const double *dvec);
int direct_apply(Engine &e, const double *b, double *x);
int direct_solve(Engine &e, double h, const double *dvec, const double *rhs, double *x);
int direct_stats(const Engine &e, long *factorizations, long *perturbed, double *flops, long *front_doubles,
                 int *fronts, int *depth);
void direct_free(Engine &e);

bool fused_supported(const Engine &e);
int fused_alloc(Engine &e, int ns);
void fused_free(Engine &e);
// With defer, the launch is not waited for: the statuses stay in
// d_fstatus[4 (slot + s) ...] ([0] iterations [1] converged [2] residual
// [3] non-finite) for the caller to read; conv is not written.
int fused_gmres(Engine &e, int ns, const double *h, const double *const *dvec, const double *const *rhs,
                double *const *x, const Cluster *const *pcs, int *conv, bool defer = false, int slot = 0);

int learned_set_weights(Engine &e, const unsigned short *bf16, long count);
int learned_build(Engine &e, double h, const double *dvec, const double *x, bool analytic);
void learned_apply_add(Engine &e, const double *v, double *z);
bool learned_rescale(Engine &e, double h, const double *dvec);
bool learned_remap(Engine &e, double h, const double *dvec);
void learned_counts(Engine &e, long *inferences, long *rescales, long *remaps);
void learned_invalidate(Engine &e);
int learned_export(Engine &e, float *host, long cap);
void learned_free(Engine &e);
long learned_weight_count();
int learned_ensure(Engine &e);
// training of the learned correction on the device (learned_train.cu)
int learned_train_init(Engine &e, const float *W0, long count);
int learned_train_step(Engine &e, double h, int k, double lr, unsigned long long seed, bool apply, double *loss,
                       float *grad);
int learned_train_weights(Engine &e, float *W, long count);
void learned_train_free(void *p);

// eigenvalue analysis (ev.cu)
int ev_hessian(Engine &e, const double *x);
const double *ev_hessian_ptr(Engine &e);
int ev_analyze(Engine &e, const double *x, const double *v, bool deriv, double rate, int corr_bins);
const double *ev_vectors(Engine &e);
const double *ev_values(Engine &e);
const double *ev_observables(Engine &e);
const double *ev_correlations(Engine &e);
void ev_timings(Engine &e, double *ms);
void ev_free(Engine &e);

} // namespace sd
