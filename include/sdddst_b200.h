/*
 * sdddst_b200 -- C ABI of the B200 (sm_100a) implicit-step engine.
 *
 * Plain pointers and sizes only; every call returns an int status
 * (SDDDST_OK = 0, negative on error; sdddst_last_error() describes the last
 * failure on the calling thread).  Unlike the reference, which ignores the
 * UMFPACK status (src/simulation.cpp:388-395, cast to void), no status is
 * dropped.  One context is driven by one host thread; it owns one CUDA stream
 * and all device memory of one simulated system.
 *
 * Configuration arrays use the reference's layouts: dislocations as N rows of
 * {x, y, b} doubles (include/dislocation.h:27-31), point defects as P rows of
 * {x, y} (include/point_defect.h:27-30).  Host pointers unless a name says
 * "_device".  Host configuration arrays must be finite: every entry point
 * that takes one checks it on the host before any device work and returns
 * SDDDST_ERR_NONFINITE for a NaN or Inf (the reference carries such values
 * into its velocities and accepts the step).
 */
#ifndef SDDDST_B200_H
#define SDDDST_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define SDDDST_OK 0
#define SDDDST_ERR_INVALID (-1)   /* bad argument or size */
#define SDDDST_ERR_CUDA (-2)      /* CUDA runtime error (message in sdddst_last_error) */
#define SDDDST_ERR_NOMEM (-3)     /* device or host allocation failed */
#define SDDDST_ERR_SOLVER (-4)    /* linear solve did not reach its tolerance */
#define SDDDST_ERR_CAPACITY (-5)  /* caller buffer too small (required size returned) */
#define SDDDST_ERR_NONFINITE (-6) /* NaN/Inf in a state or result */

/* StressProtocol family: getType() "zero-stress" (stress_protocol.cpp:54-57),
 * "fixed-rate-stress" (fixed_rate_protocol.cpp:80-83), "spring-stress"
 * (spring_protocol.cpp:56-59), and a constant value (any other type string). */
enum {
    SDDDST_STRESS_ZERO = 0,
    SDDDST_STRESS_FIXED_RATE = 1,
    SDDDST_STRESS_SPRING = 2,
    SDDDST_STRESS_CONSTANT = 3
};

/* StressProtocolStepType (stress_protocol.h:31-37). */
enum {
    SDDDST_STAGE_ORIGINAL = 0,
    SDDDST_STAGE_END_OF_BIG_STEP = 1,
    SDDDST_STAGE_END_OF_FIRST_SMALL_STEP = 2,
    SDDDST_STAGE_END_OF_SECOND_SMALL_STEP = 3
};

/* Arithmetic of the O(N^2) pair sum. */
enum {
    SDDDST_PAIRSUM_FP64 = 0, /* plain: FP64 throughout */
    SDDDST_PAIRSUM_FP32 = 1  /* FP32 pair terms, FP64 (compensated) accumulation */
};

/* Linear solver replacing UMFPACK (simulation.cpp:386-396). */
enum {
    SDDDST_SOLVER_GMRES = 0,         /* restarted GMRES, FP64, unpreconditioned */
    SDDDST_SOLVER_GMRES_JACOBI = 1,  /* restarted GMRES, FP64, diagonal preconditioner */
    SDDDST_SOLVER_GMRES_CLUSTER = 2, /* restarted GMRES, FP64, block-Jacobi on strongly coupled clusters */
    SDDDST_SOLVER_DIRECT = 3,        /* sparse LU (multifrontal, nested dissection), FP64, refined to solver_tol */
    SDDDST_SOLVER_GMRES_LEARNED = 4, /* restarted GMRES, FP64, cluster block-Jacobi plus a learned correction on
                                        J's pattern (weights: sdddst_set_preconditioner_weights); falls back to
                                        the sparse LU when GMRES stalls */
    SDDDST_SOLVER_GMRES_NEUMANN = 5, /* as SDDDST_SOLVER_GMRES_LEARNED with the analytic first-order
                                        block-Neumann correction in place of the network */
    SDDDST_SOLVER_DIRECT_MIXED = 6   /* sparse LU with FP32 fronts, FP64 iterative refinement to solver_tol */
};

/* Field kernels (Field plug-in): the analytic periodic field
 * (Fields/AnalyticField.cpp). */
enum {
    SDDDST_FIELD_ANALYTIC = 0,  /* AnalyticField (AnalyticField.cpp:145-181) */
    SDDDST_FIELD_TABULATED = 1  /* tabulated 1024 x 1024 field with bicubic interpolation, the counterpart of
                                   PeriodicShearStressELTE (python/src/periodic_shear_stress_ELTE_wrapper.cpp:40-46);
                                   tables built on the device from the analytic field; FP64 pair sum */
};

typedef struct {
    int n;                    /* dislocation count (SimulationData::dc) */
    int p;                    /* point-defect count (SimulationData::pc) */
    double cutoff_multiplier; /* SimulationData::cutOffMultiplier */
    double prec;              /* SimulationData::prec */
    double step_size;         /* SimulationData::stepSize (initial) */
    double A;                 /* SimulationData::A (after any scaling) */
    double KASQR;             /* SimulationData::KASQR (after any scaling) */
    int ic;                   /* SimulationData::ic, chord-Newton iterations */
    int stress_kind;          /* SDDDST_STRESS_* */
    double stress_rate;       /* FixedRateProtocol::rate */
    double spring_constant;   /* SpringProtocol::springConstant */
    double stress_value;      /* constant protocol */
    int calculate_strain;     /* SimulationData::calculateStrainDuringSimulation */
    int max_step_limited;     /* SimulationData::isMaxStepSizeLimit */
    double max_step;          /* SimulationData::maxStepSizeLimit */
    int field;                /* SDDDST_FIELD_* */
    int pairsum;              /* SDDDST_PAIRSUM_* */
    int solver;               /* SDDDST_SOLVER_* */
    double solver_tol;        /* relative residual target of the iterative solve */
    int gmres_restart;        /* Krylov subspace size per cycle */
    int max_iters;            /* iteration cap per solve */
    double precond_theta;     /* coupling strength that joins two dislocations in a cluster
                                 (0: 0.01 for SDDDST_SOLVER_GMRES_CLUSTER, 0.05 under the learned
                                 and analytic corrections) */
    int device;               /* CUDA device ordinal */
    double neumann_theta;     /* SDDDST_SOLVER_GMRES_NEUMANN: cross-block couplings of normalised strength
                                 |A_ij| / sqrt(|J_ii J_jj|) below this are left out of the correction */
} sdddst_params;

/* Defaults of SimulationData() (simulation_data.cpp:43-109, constants.h):
 * cutoff multiplier 1, prec 1e-8, step 1, A = 1.6e-3, KASQR = 1.65^2*1e6/256,
 * ic = 2, zero stress, FP64 pair sum, cluster-preconditioned GMRES (coupling
 * threshold 0.01, at most 300 iterations, then retried with a rebuilt
 * preconditioner) to 1e-13. */
void sdddst_default_params(sdddst_params *prm);

/* Creates a context and uploads the configuration.  Replaces constructing
 * SimulationData + Simulation (simulation_data.cpp:111-117,
 * simulation.cpp:38-55); the cutoff follows SimulationData::updateCutOff
 * (simulation_data.cpp:208-218). */
int sdddst_ctx_create(const sdddst_params *prm, const double *xyb, const double *pd, void **ctx);
int sdddst_ctx_destroy(void *ctx);

/* Error text of the last failing call on this thread. */
const char *sdddst_last_error(void);

/* Replaces the state: positions, step size, time, energy, strain.  With
 * first_step = 0 the state is taken as just accepted (initial velocities
 * re-evaluated as at simulation.cpp:543-550, tolerances reset as at :644);
 * with first_step = 1 the next step behaves as a fresh Simulation's first
 * step (simulation.cpp:450-479). */
int sdddst_set_state(void *ctx, const double *xyb, double step_size, double sim_time, double energy,
                     double strain, int first_step);

/* Scalars after the last step, same order as the oracle:
 * [0] simTime [1] stepSize [2] successful steps [3] failed steps [4] energy
 * [5] accumulated strain [6] max error ratio^2 of the last attempt
 * [7] <|v|> [8] sum v^2 [9] energy increment [10] cutoff [11] stress(Original) */
int sdddst_get_scalars(void *ctx, double *out12);

/* which: 0 accepted configuration, 1 big step, 2 first small step,
 * 3 second small step; writes N x {x, y, b}. */
int sdddst_get_config(void *ctx, int which, double *xyb);

/* which: 0 initSpeed, 1 initSpeed2, 2 speed, 3 speed2, 4 dVec, 5 g,
 * 6 tolerance at the end of the last step (before its reset). */
int sdddst_get_vector(void *ctx, int which, double *out);

/* Simulation::calculateSpeeds (simulation.cpp:86-131) on a given
 * configuration with a fresh precision handler: velocities v[N] and the
 * per-dislocation tolerance tol[N] (precision_handler.cpp:72-87).
 * stress_type selects the stored stress value (after calculateStress at
 * sim_time for that step type). */
int sdddst_speeds(void *ctx, const double *xyb, double sim_time, int stress_type, double *v, double *tol);

/* calculateSpeeds with an explicit external stress: v[N] = pair sum + point
 * defects + b tau_ext on the given configuration, and minr2[N], the
 * smallest distance measure each dislocation saw (r^2 to dislocations,
 * X2(dx)+X2(dy) to point defects) among those below 400 prec^2 (+inf
 * otherwise) -- the argument the reference passes to
 * PrecisionHandler::updateTolerance (precision_handler.cpp:72-87). */
int sdddst_speeds_ext(void *ctx, const double *xyb, double tau_ext, double *v, double *minr2);

/* Replaces the step state scalars without touching the configuration:
 * SimulationData::stepSize, simTime, totalAccumulatedStrainIncrease and the
 * Simulation's accumulated energy. */
int sdddst_set_scalars(void *ctx, double step_size, double sim_time, double energy, double strain);

/* Updates the mutable parameters of a live context from prm (cutoff
 * multiplier with SimulationData::updateCutOff, precision, max step size,
 * stress protocol parameters, solver settings); sizes and the field kind
 * must be unchanged. */
int sdddst_update_params(void *ctx, const sdddst_params *prm);

/* Solves A x = b for a general N x N matrix given in CSC (Ap[N+1], Ai, Ax:
 * UMFPACK's layout, as the reference's solveEQSys passes it,
 * simulation.cpp:393-396) with the context's device solver.  The context's
 * assembled Jacobian is replaced (the next step reassembles). */
int sdddst_solve_csc(void *ctx, const int *Ap, const int *Ai, const double *Ax, const double *b, double *x,
                     int *iterations);

/* Simulation::calculateJacobian (simulation.cpp:236-384) at step size h on a
 * given configuration, returned as CSR of J (row i = dislocation i; the
 * reference's CSC column j is row j of J^T).  row_ptr[N+1], col[cap],
 * val[cap], dvec[N].  On SDDDST_ERR_CAPACITY, *nnz holds the size needed. */
int sdddst_jacobian(void *ctx, double h, const double *xyb, int *row_ptr, int *col, double *val, double *dvec,
                    long cap, long *nnz);

/* Solves J(h, xyb) x = rhs with the context's solver (the UMFPACK
 * symbolic + numeric + solve sequence, simulation.cpp:386-396). */
int sdddst_solve(void *ctx, double h, const double *xyb, const double *rhs, double *x, int *iterations);

/* Simulation::step (simulation.cpp:435-441): one adaptive implicit step
 * (full step, two half steps, error control, accept/reject, new step size). */
int sdddst_step(void *ctx, int *accepted);

/* Repeats sdddst_step until `accepted_target` steps were accepted or
 * `max_attempts` attempts were made. */
int sdddst_run(void *ctx, int accepted_target, int max_attempts, int *accepted, int *attempts);

/* Device-resident access for callers that keep the state on the GPU:
 * pointers to the accepted configuration's x, y and b arrays (N doubles each,
 * structure of arrays) on the context's device. */
int sdddst_state_device(void *ctx, double **x_device, double **y_device, double **b_device);

/* Replaces the accepted configuration's x coordinates (N doubles, host)
 * without re-evaluating the initial velocities: for round trips of a state
 * the context already holds (y, b and the step state are unchanged).  With
 * recompute = 1 the initial velocities are re-evaluated as after an accepted
 * step (simulation.cpp:543-550). */
int sdddst_upload_positions(void *ctx, const double *x, int recompute);

/* Copies the accepted configuration's x coordinates (N doubles) to the host. */
int sdddst_download_positions(void *ctx, double *x);

/* The context's CUDA stream (a cudaStream_t), for callers that time or
 * order work against it. */
int sdddst_stream(void *ctx, void **stream);

/* Roofline denominators of the CUDA-core pipes on `device`: sustained FP64
 * and FP32 fused multiply-add throughput in TFLOP/s (2 FLOP per FMA),
 * measured by a short dependent-chain microbenchmark (~0.1 s). */
int sdddst_vector_peaks(int device, double *fp64_tflops, double *fp32_tflops);

/* Times `reps` back-to-back launches of the pair-sum kernels on the accepted
 * configuration with CUDA events on the context's stream; writes the mean
 * device time of one launch (tile kernel and its min-distance reset). */
int sdddst_profile_pair_sum(void *ctx, int reps, double *ms_per_launch);

/* Allocation-free velocity evaluation, for callers that cannot allocate
 * device memory (their memory is budgeted by another framework, or a
 * cudaMalloc and its implicit device-wide synchronisation would stall the
 * work they interleave with).  No counterpart in the reference.
 *
 * Computes v_i = sum_{j != i} b_i b_j tau_xy(x_i - x_j, y_i - y_j) + b_i tau_ext
 * (the pair sum of calculateSpeeds without point defects or tolerances) in
 * FP64, the same kernels as sdddst_speeds.  Inputs x, y, b and the output v
 * are N doubles each in device memory; the work is queued on `stream`
 * (a cudaStream_t, NULL for the default stream) and not synchronised.
 *
 * Scratch: a static 2 MiB __device__ array inside this library, held by every
 * GPU that loads the library until the process exits; N is limited to 4096
 * (larger N returns SDDDST_ERR_CAPACITY).  The first call on each device
 * looks up the array's device address (with that device current); make that
 * first call before any stream capture.  No cudaMalloc, cudaFree or other
 * allocating call is made.  All calls share the one array, which keeps the
 * last call's contents: calls that overlap on the GPU (different streams, or
 * host threads using the same device) race and must be serialised by the
 * caller.  Every scratch slot is written before it is read, so nothing needs
 * clearing between calls.  The looked-up address is cached per device for
 * the life of the process: after cudaDeviceReset (or any destruction of the
 * device's primary context) in the calling process the cached address is
 * stale and this entry point must not be called again. */
int sdddst_speeds_noalloc(int n, const double *x_device, const double *y_device, const double *b_device,
                          double tau_ext, double *v_device, void *stream);

/* Linear-solver statistics of this context: solves performed and their
 * total Krylov iterations. */
int sdddst_solver_stats(void *ctx, long *solves, long *iterations);

/* Recoveries in this context (each pointer optional): rebuilds counts
 * cluster-preconditioner rebuilds with a five times lower coupling threshold
 * after a stalled solve (GMRES past max_iters; SDDDST_SOLVER_GMRES_CLUSTER,
 * at most two per solve before SDDDST_ERR_SOLVER), fallbacks counts
 * learned- or analytic-corrected solves redone by the sparse LU, and redone
 * counts step attempts of the cluster solver that ran without waiting for the
 * device, failed a deferred check (a stalled solve, a pattern larger than the
 * Jacobian storage) and were repeated with a wait at every check.  The
 * reference has none of these: its UMFPACK status is ignored
 * (simulation.cpp:388-395). */
int sdddst_solver_recoveries(void *ctx, long *rebuilds, long *fallbacks, long *redone);

/* ---- eigenvalue analysis: the reference's --ev-analyzation mode
 * (src/main.cpp:36-41; TimeSeriesProcessor::run, src/time_series_processor.cpp:21-204;
 * SpectralDecompositor::decompose, src/spectral_decompositor.cpp:63-201).
 * The context supplies n, the point defects and the stress protocol; xyb is
 * the configuration (n x 3, x y b).  The Hessian's defect term uses the
 * decomposer's own scaling, A = 1.6e-3 / sqrt(defect count) and
 * K = 1.65^2 1e6 / 256 * n (spectral_decompositor.cpp:76-84); the velocities
 * use the context's A and KASQR (DataTimeSeries::next sets A = 1.6e-3 /
 * sqrt(n), KASQR = 1.65^2 1e6 / 256 * n, data_time_series.cpp:34-35). */

/* The dense Hessian decompose() hands to LAPACKE_dsyevd: H (n x n,
 * symmetric) with H_ij = b_i b_j xy_diff_x(x_i - x_j, y_i - y_j) off the
 * diagonal and H_ii = -sum_{j != i} H_ij - b_i sum_defects d/dx(defect force). */
int sdddst_ev_hessian(void *ctx, const double *xyb, double *H);

/* One configuration of TimeSeriesProcessor::run.  Every output may be NULL:
 *   eigenvalues    n, ascending (getEigenValue)
 *   participation  n, 1 / sum_j v_mj^4                         (:46-53)
 *   burgers_sum    n, s_m = sum_j v_mj b_j                      (:77-84)
 *   gan            n, s_m^2 / lambda_m                          (:55-62)
 *   speeds         n, calculateSpeeds at sim_time, stress Original (:64-68)
 *   eigenvectors   nvec x n (eigenvector m contiguous), nvec <= n (:86-91)
 *   derivatives    n, eigenvalue derivatives (:93-121) under a fixed-rate
 *                  protocol; zeros under any other, as in the reference
 *   correlations   n x 3 x S x S: per mode the equal-sign, opposite-sign and
 *                  all-pairs histograms of (:145-197), S = corr_bins
 * Eigenvector signs are those of the device eigensolver (any sign is an
 * eigenvector; the sign-free outputs do not depend on it). */
int sdddst_ev_analyze(void *ctx, const double *xyb, double sim_time, double *eigenvalues, double *participation,
                      double *burgers_sum, double *gan, double *speeds, double *eigenvectors, int nvec,
                      double *derivatives, double *correlations, int corr_bins);

/* Device times (ms, CUDA events) of the last sdddst_ev_analyze: Hessian,
 * eigensolver, observables, derivatives, correlation matrices. */
int sdddst_ev_timings(void *ctx, double *ms5);

/* Sparse LU statistics of this context (SDDDST_SOLVER_DIRECT; zeros
 * otherwise): factorizations performed, pivots perturbed, FP64 flops of one
 * factorization of the last analysed pattern, doubles held by its fronts,
 * number of fronts and tree depth (each pointer optional).  The reference
 * reports nothing comparable: UMFPACK's statistics are not read
 * (simulation.cpp:386-396). */
int sdddst_direct_stats(void *ctx, long *factorizations, long *perturbed, double *flops, long *front_doubles,
                        int *fronts, int *depth);

/* Diagnostic timing of the sparse LU (SDDDST_SOLVER_DIRECT contexts): the
 * Jacobian J(h) at the accepted configuration is assembled and analysed,
 * factored once untimed, then factored `reps` times and solved `reps` times
 * with CUDA events on the context's stream; writes the mean device
 * milliseconds of one factorization and of one forward/backward solve.
 * Stands in for timing UMFPACK's numeric factorization and solve
 * (simulation.cpp:386-396). */
int sdddst_profile_direct(void *ctx, double h, int reps, double *factor_ms, double *solve_ms);

/* Applies the cluster block-Jacobi preconditioner of J(h) at the accepted
 * configuration to k device vectors (in_device, out_device: k x n doubles,
 * vector q at offset q n) and, when block_of_device is not null, writes each
 * dislocation's block index (n ints, device).  Produces the training data of
 * the learned preconditioner; no counterpart in the reference. */
int sdddst_precond_apply(void *ctx, double h, int k, const double *in_device, double *out_device,
                         int *block_of_device);

/* Weights of the learned preconditioner correction (SDDDST_SOLVER_GMRES_LEARNED):
 * `count` BF16 bit patterns in the flat order of sdddst_b200/learned.py
 * (59522 for the shipped network); SDDDST_ERR_INVALID on another count.  No
 * counterpart in the reference. */
int sdddst_set_preconditioner_weights(void *ctx, const unsigned short *bf16, long count);

/* The learned correction C for J(h) at the accepted configuration: `nnz`
 * floats aligned with the CSR of sdddst_jacobian (diagonal in each row's
 * first slot).  Requires loaded weights; no counterpart in the reference. */
int sdddst_learned_correction(void *ctx, double h, float *values, long cap, long *nnz);

/* Training of the learned correction on the device (the network of
 * sdddst_set_preconditioner_weights): hand-written forward and backward
 * kernels, node products and weight gradients on the tensor cores (BF16
 * operands, FP32 accumulation), Adam on FP32 master weights with global-norm
 * clipping at 1; the BF16 weights the inference reads follow every step.
 * The context should use SDDDST_SOLVER_GMRES_LEARNED (its cluster
 * threshold is the one the correction is trained against).
 *   init:    FP32 starting weights (count = the flat weight count);
 *   step:    the Jacobian J(h) at the context's accepted configuration, its
 *            cluster inverse B and `probes` (1..8) random sign probes Z from
 *            `seed`: loss2[0] = ||Z - J B Z||^2 / ||Z||^2 (B alone),
 *            loss2[1] = ||Z - J (B + C) Z||^2 / ||Z||^2 (the loss), both
 *            before the update; with apply, one Adam step at rate lr on
 *            the ratio loss2[1] / loss2[0] (scale-free across step sizes);
 *            grad (optional, count floats) the gradient of that ratio;
 *   weights: the FP32 master weights. */
int sdddst_learned_train_init(void *ctx, const float *weights, long count);
int sdddst_learned_train_step(void *ctx, double h, int probes, double lr, unsigned long long seed, int apply,
                              double *loss2, float *grad);
int sdddst_learned_train_weights(void *ctx, float *weights, long count);

/* ---- Batches of independent systems (a population of random realisations).
 * `count` systems of sizes[k] dislocations, concatenated in xyb (sum of sizes
 * rows of {x, y, b}), share the parameters of `common` (n, p and the stress
 * protocol are ignored: every system has no point defects and zero external
 * stress).  Each system keeps its own cutoff (multiplier / sqrt(N_k)), step
 * size, time, energy and counters and accepts or rejects its own steps
 * (Simulation::step, simulation.cpp:435-650, per system); every phase of a
 * step is one launch over all systems. */
int sdddst_batch_create(const sdddst_params *common, int count, const int *sizes, const double *xyb, void **batch);
int sdddst_batch_destroy(void *batch);
/* One step attempt of every system; accepted[k] (optional, count ints)
 * receives 1 where system k accepted. */
int sdddst_batch_step(void *batch, int *accepted);
/* count x 12 scalars, the layout of sdddst_get_scalars (entries without a
 * batched counterpart are 0). */
int sdddst_batch_get_scalars(void *batch, double *out);
/* x coordinates of all systems (which: 0 accepted, 1 big step, 2 first small
 * step, 3 second small step), sum of sizes doubles. */
int sdddst_batch_get_positions(void *batch, int which, double *x);
/* Pair-sum tile chosen by the autotuner, total dislocations, kernels launched
 * so far and the batch's cudaStream_t (each pointer optional). */
int sdddst_batch_info(void *batch, int *tile, long *total, long *launches, void **stream);

/* How the batch steps (each pointer optional): *graph = 1 when its steps
 * after the first replay one captured CUDA graph (no host round trip until
 * the step's end), 0 when they are enqueued directly or host-driven;
 * *redone counts steps whose deferred checks failed (a stalled solve, a
 * pattern larger than the Jacobian storage, a non-finite error ratio) and
 * were repeated host-driven from the step's snapshot. */
int sdddst_batch_stats(void *batch, int *graph, long *redone);

/* Times `reps` launches of the batch's pair-sum kernel (all systems' tiles,
 * FP32 or FP64 as created) on the accepted configurations with CUDA events
 * on the batch's stream; writes the mean device milliseconds of one launch
 * and the number of unique pairs it evaluates. */
int sdddst_batch_profile_pair_sum(void *batch, int reps, double *ms_per_launch, double *pairs);

/* Launch statistics: number of kernels this context has launched so far. */
long sdddst_kernel_launches(void *ctx);

#ifdef __cplusplus
}
#endif

#endif
