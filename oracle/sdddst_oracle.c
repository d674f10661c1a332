/*
 * CPU restatement of SDDDST's implicit-step hot path (the oracle).
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py load this library, as the checker of the CUDA
 * path; the product never links or calls it.
 *
 * It restates, in plain C and in the same floating-point operation order,
 * the reference algorithm of pgabor/sdddst:
 *   field kernels      src/Fields/AnalyticField.cpp:24-181 (f, g, f_dx, g_dx,
 *                      AnalyticField::xy, ::xy_diff_x), ANALYTIC_FIELD_N = 4
 *                      (include/constants.h:25)
 *   helpers            include/utility.h:29-50,92-100 (normalize, X, X2,
 *                      calculateStrainIncrement)
 *   precision handler  src/precision_handler.cpp:62-119
 *   velocities         src/simulation.cpp:86-131 (calculateSpeeds)
 *   residual           src/simulation.cpp:133-193 (calculateG)
 *   Jacobian           src/simulation.cpp:236-384 (calculateJacobian); the CSC
 *                      is built row-wise from the symmetric H and scaled, which
 *                      gives the same pattern, values and summation order
 *   solve              src/simulation.cpp:386-396 through the UMFPACK shim
 *   integrate / step   src/simulation.cpp:62-84,398-415,435-650
 * and the CLI's set-up of SimulationData (src/project_parser.cpp:137-298,
 * src/simulation_data.cpp:43-109,208-218); for the eigenvalue analysis the
 * second field derivative (AnalyticField.cpp:95-132,183-202), the Hessian
 * (src/spectral_decompositor.cpp:63-165), the eigenvalue derivatives and the
 * correlation matrices (src/time_series_processor.cpp:104-197,208-247).
 *
 * Its exported calls have the same names and meaning as oracle/ref_harness.cpp
 * so that one Python wrapper (oracle/ref.py) drives either library; tests pin
 * this restatement against the compiled reference and the golden fixtures.
 */
#include "umfpack.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif
#ifndef M_E
#define M_E 2.7182818284590452354
#endif

#define ORC_EPS 1e-12 /* constants.h:24 */
#define ORC_FIELD_N 4 /* constants.h:25 */

double orc_xy_diff_x2(double dx, double dy);

/* ------------------------------------------------------------ helpers --- */

/* utility.h:29-40 */
static inline void normalize(double *n)
{
    while (*n < -0.5) *n += 1.0;
    while (*n >= 0.5) *n -= 1.0;
}

/* utility.h:42-50 */
static inline double Xf(double x) { return sin(2.0 * M_PI * x) * 0.5 / M_PI; }
static inline double X2f(double x) { return (1.0 - cos(2.0 * M_PI * x)) * 0.5 / M_PI / M_PI; }

/* ------------------------------------------------------- field kernels --- */

/* AnalyticField.cpp:24-39: tau_xy of one y-periodic column of images; Taylor
 * branch of cosh-1, cos-1 and cosh-cos when dx^2+dy^2 <= 1e-6. */
static double fpair(double dx, double cos2piy, double dy)
{
    if (dx * dx + dy * dy > 1e-6) {
        double c = cosh(dx * 2.0 * M_PI);
        return dx * (c * cos2piy - 1.0) / ((c - cos2piy) * (c - cos2piy)) * 2. * M_PI * M_PI;
    }
    double a = dx * 2.0 * M_PI;
    double b = dy * 2.0 * M_PI;
    double a2 = pow(a, 2), a4 = pow(a, 4.0), a6 = pow(a, 6.0);
    double b2 = pow(b, 2), b4 = pow(b, 4), b6 = pow(b, 6.0);
    double chm1 = a6 / 720.0 + a4 / 24.0 + a2 * 0.5;
    double cm1 = -b6 / 720.0 + b4 / 24.0 - b2 * 0.5;
    double cmc = (b6 + a6) / 720. + (a4 - b4) / 24.0 + (a2 + b2) * 0.5;
    return ((chm1 * cm1 + cm1 + chm1) * dx) / (pow(cmc, 2.0)) * 2.0 * pow(M_PI, 2.0);
}

/* AnalyticField.cpp:41-51: image sum g<images> = f(dx) + sum_k f(dx-k)+f(dx+k),
 * accumulated in the template's order. */
static double gimg(int images, double dx, double cos2piy, double dy)
{
    double s = fpair(dx, cos2piy, dy);
    for (int k = 1; k <= images; ++k)
        s = s + fpair(dx - (double)k, cos2piy, dy) + fpair(dx + (double)k, cos2piy, dy);
    return s;
}

/* AnalyticField.cpp:53-93: d/dx of fpair.  The Taylor series of
 * sinh(a)cos(b) keeps the reference's a^7 b^2 coefficient 1/1080 (the exact
 * series has 1/10080; the term is below 1e-17 relative inside the branch). */
static double fpair_dx(double dx, double cos2piy, double dy)
{
    double c = cosh(M_PI * 2.0 * dx);
    double s = sinh(M_PI * 2.0 * dx);
    if (dx * dx + dy * dy > 1e-6) {
        return ((c * cos2piy - 1.0) / pow(c - cos2piy, 2.0) +
                dx * (s * cos2piy * 2.0 * M_PI / pow(c - cos2piy, 2.0) -
                      (c * cos2piy - 1.0) / pow(c - cos2piy, 3.0) * 4.0 * M_PI * s)) *
               M_PI * M_PI * 2.0;
    }
    double a = dx * 2.0 * M_PI;
    double b = dy * 2.0 * M_PI;
    double a2 = pow(a, 2), a3 = pow(a, 3.0), a4 = pow(a, 4.0), a5 = pow(a, 5.0), a6 = pow(a, 6.0),
           a7 = pow(a, 7.0);
    double b2 = pow(b, 2.0), b4 = pow(b, 4.0), b6 = pow(b, 6.0);
    double chm1 = a6 / 720.0 + a4 / 24.0 + a2 * 0.5;
    double cm1 = -pow(b, 6.0) / 720.0 + pow(b, 4) / 24.0 - pow(b, 2) * 0.5;
    double cmc = (b6 + a6) / 720. + (a4 - b4) / 24.0 + (pow(a, 2.0) + b2) * 0.5;
    double sc = -(a7 * b6) / 3628800.0 - (a5 * b6) / 86400.0 - (a3 * b6) / 4320.0 - (b6 * a) / 720 +
                (a7 * b4) / 120960.0 + (a5 * b4) / 2880.0 + (a3 * b4) / 144.0 + (b4 * a) / 24.0 -
                (a7 * b2) / 1080.0 - (a5 * b2) / 240.0 - (a3 * b2) / 12.0 - (b2 * a) * 0.5 +
                a7 / 5040.0 + a5 / 120.0 + a3 / 6.0 + a;
    double num = chm1 * cm1 + cm1 + chm1;
    return (num / pow(cmc, 2.0) +
            ((sc * dx) / (pow(cmc, 2.0)) - num / (pow(cmc, 3.0)) * dx * sinh(a) * 2.0) * M_PI * 2.0) *
           2.0 * pow(M_PI, 2.0);
}

/* AnalyticField.cpp:110-120 */
static double gimg_dx(int images, double dx, double cos2piy, double dy)
{
    double s = fpair_dx(dx, cos2piy, dy);
    for (int k = 1; k <= images; ++k)
        s = s + fpair_dx(dx - (double)k, cos2piy, dy) + fpair_dx(dx + (double)k, cos2piy, dy);
    return s;
}

/* AnalyticField::xy, AnalyticField.cpp:145-160: explicit x-images |k| <= 3,
 * f(dx -/+ 4) and the linearly weighted end images. */
double orc_xy(double dx, double dy)
{
    const double n = (double)ORC_FIELD_N;
    double cy = cos(M_PI * 2.0 * dy);
    if (dx < 0)
        return -dx * fpair(dx + (double)(ORC_FIELD_N + 1), cy, dy) + (1.0 + dx) * fpair(dx - n, cy, dy) +
               fpair(dx + n, cy, dy) + gimg(ORC_FIELD_N - 1, dx, cy, dy);
    return dx * fpair(dx - ((double)(ORC_FIELD_N + 1)), cy, dy) + (1.0 - dx) * fpair(dx + n, cy, dy) +
           fpair(dx - n, cy, dy) + gimg(ORC_FIELD_N - 1, dx, cy, dy);
}

/* AnalyticField::xy_diff_x, AnalyticField.cpp:162-181 */
double orc_xy_diff_x(double dx, double dy)
{
    const double n = (double)ORC_FIELD_N;
    double cy = cos(M_PI * 2.0 * dy);
    if (dx < 0)
        return -fpair(dx + n + 1.0, cy, dy) - dx * fpair_dx(dx + n + 1.0, cy, dy) +
               fpair_dx(dx - n, cy, dy) * (1.0 + dx) + fpair(dx - n, cy, dy) + fpair_dx(dx + n, cy, dy) +
               gimg_dx(ORC_FIELD_N - 1, dx, cy, dy);
    return fpair(dx - n - 1.0, cy, dy) + dx * fpair_dx(dx - n - 1.0, cy, dy) +
           fpair_dx(dx + n, cy, dy) * (1.0 - dx) - fpair(dx + n, cy, dy) + fpair_dx(dx - n, cy, dy) +
           gimg_dx(ORC_FIELD_N - 1, dx, cy, dy);
}

/* d/dx of the point-defect force divided by b, i.e. of
 * -2 A X(dx) X(dy) ((1-e^{-K s})/s - K e^{-K s})/s with s = X2(dx)+X2(dy);
 * the reference writes it out term by term inside calculateJacobian
 * (simulation.cpp:288-322).  Same three terms, same grouping. */
static double pd_force_dx(double dx, double dy, double A, double K)
{
    double cx = cos(2.0 * M_PI * dx), sx = sin(2.0 * M_PI * dx);
    double sy = sin(2.0 * M_PI * dy), cyy = cos(2.0 * M_PI * dy);
    double s = (1.0 - cx) * pow(M_PI, -2.0) / 2.0 + (1.0 - cyy) * pow(M_PI, -2.0) / 2.0;
    double e = pow(M_E, -K * s); /* the reference writes e^x as pow(M_E, x) here */
    double le = log(M_E);
    double phi = ((1.0 - e) / s - K * e);
    double t1 = -A * cx / M_PI * sy * phi / s;
    double t2 = -A * sx * pow(M_PI, -2.0) * sy *
                (e * K * sx / M_PI * le / s - (1.0 - e) * pow(s, -2.0) * sx / M_PI + K * K * e * sx / M_PI * le) /
                s / 2.0;
    double t3 = A * pow(sx, 2.0) * pow(M_PI, -3.0) * sy * phi * pow(s, -2.0) / 2.0;
    return t1 + t2 + t3;
}

/* ---------------------------------------------------------- simulation --- */

typedef struct {
    double cutoff_multiplier, prec, step_size;
    int stress_kind;
    double stress_rate, spring_constant, stress_value;
    int pd_scaling, calculate_strain, order_parameter, max_step_limited;
    double max_step;
} ref_params;

enum { ST_ORIGINAL = 0, ST_END_BIG = 1, ST_END_FIRST = 2, ST_END_SECOND = 3 };

typedef struct {
    int n, p;
    double *x, *y, *b;     /* accepted configuration (dislocations) */
    double *xb, *x1, *x2;  /* bigStep, firstSmall, secondSmall (x only: y, b never change) */
    double *pdx, *pdy;
    double *v0, *v0b, *vs, *vs2, *g, *dvec, *sol;
    double *tol, *errv;    /* precision handler: tolerance, error */
    double max_ratio, last_ratio;
    double *last_tol;
    /* parameters (SimulationData) */
    double cutoff_multiplier, cutoff, cutoff_sqr, one_per_cutoff_sqr, prec, prec_sqr;
    double A, KASQR, step_size, sim_time, strain;
    int ic, stress_kind, calc_strain, order_param, max_step_limited;
    double stress_rate, spring_k, stress_value, max_step;
    double stress_vals[4];
    int cur_stress;
    /* Simulation members */
    int first_step, init_speed_needed, successful_step;
    double energy, energy_accum, vsquare, vsquare1, vsquare2, sum_avg_speed;
    long succ, failed;
    /* CSC Jacobian */
    int *Ap, *Ai;
    double *Ax;
    long cap;
    void *numeric;
} orc_sim;

static double *dalloc(int n) { return (double *)calloc((size_t)(n > 0 ? n : 1), sizeof(double)); }

/* simulation_data.cpp:208-218 */
static void update_cutoff(orc_sim *s)
{
    double m = s->cutoff_multiplier;
    if (s->cutoff_multiplier >= 1. / 12. * sqrt(2.0 * (double)s->n)) m = 1e20;
    s->cutoff = 1. / sqrt((double)s->n) * m;
    s->cutoff_sqr = s->cutoff * s->cutoff;
    s->one_per_cutoff_sqr = 1. / s->cutoff_sqr;
}

/* precision_handler.cpp:62-70 */
static void ph_reset(orc_sim *s)
{
    s->max_ratio = 0;
    for (int i = 0; i < s->n; ++i) {
        s->tol[i] = s->prec_sqr;
        s->errv[i] = 0;
    }
}

/* precision_handler.cpp:72-87 */
static inline void ph_update_tol(orc_sim *s, double r2, int id)
{
    double t = r2 * 0.25 * 1e-2;
    if (t < s->prec_sqr && t < s->tol[id]) s->tol[id] = (t == 0.0) ? ORC_EPS : t;
}

/* precision_handler.cpp:89-101 */
static inline void ph_update_err(orc_sim *s, double e, int id)
{
    if (s->errv[id] < e) {
        s->errv[id] = e;
        double t = e * e / s->tol[id];
        if (t > s->max_ratio) s->max_ratio = t;
    }
}

/* precision_handler.cpp:103-119 */
static double ph_new_step(const orc_sim *s, double h)
{
    if (0.0 == s->max_ratio) return h * 2.0;
    double t = 1. / sqrt(s->max_ratio);
    t = pow(t, 1. / 3.);
    if (t > 2.0) t = 2.0;
    return 0.9 * h * t;
}

/* Stress protocols: stress_protocol.cpp:32-57 (zero), fixed_rate_protocol.cpp:
 * 39-73 (rate*t), spring_protocol.cpp:33-54 (k*(rate*t - strain), clamped at 0),
 * and a constant value (kind 3). */
static void stress_calc(orc_sim *s, double t, int type, double strain)
{
    if (s->stress_kind == 1) s->stress_vals[type] = t * s->stress_rate;
    else if (s->stress_kind == 2) {
        double v = s->spring_k * (t * s->stress_rate - strain);
        if (v < 0) v = 0;
        s->stress_vals[type] = v;
    }
}

static double stress_get(const orc_sim *s, int type)
{
    if (s->stress_kind == 1 || s->stress_kind == 2) return s->stress_vals[type];
    if (s->stress_kind == 3) return s->stress_value;
    return 0.0;
}

static int zero_stress(const orc_sim *s) { return s->stress_kind == 0; }

/* utility.h:92-100 */
static double strain_inc(const orc_sim *s, const double *xo, const double *xn)
{
    double r = 0;
    for (int i = 0; i < s->n; ++i) r += s->b[i] * (xn[i] - xo[i]);
    return r;
}

/* Simulation::calculateSpeeds, simulation.cpp:86-131 */
static void calc_speeds(orc_sim *s, const double *xs, double *res, int ignore_ph)
{
    int n = s->n;
    for (int i = 0; i < n; ++i) res[i] = 0;
    for (int i = 0; i < n; ++i) {
        for (int j = i + 1; j < n; ++j) {
            double dx = xs[i] - xs[j];
            normalize(&dx);
            double dy = s->y[i] - s->y[j];
            normalize(&dy);
            double t = s->b[i] * s->b[j] * orc_xy(dx, dy);
            double r2 = dx * dx + dy * dy;
            if (!ignore_ph) {
                ph_update_tol(s, r2, i);
                ph_update_tol(s, r2, j);
            }
            res[i] += t;
            res[j] -= t;
        }
        for (int j = 0; j < s->p; ++j) {
            double dx = xs[i] - s->pdx[j];
            normalize(&dx);
            double dy = s->y[i] - s->pdy[j];
            normalize(&dy);
            double xq = X2f(dx), yq = X2f(dy);
            double rq = xq + yq;
            double e = exp(-s->KASQR * rq);
            res[i] -= 2.0 * s->A * Xf(dx) * Xf(dy) * ((1. - e) / rq - s->KASQR * e) / rq * s->b[i];
            if (!ignore_ph) ph_update_tol(s, rq, i);
        }
        res[i] += s->b[i] * stress_get(s, s->cur_stress);
    }
}

/* Row-wise build of the CSC Jacobian (simulation.cpp:236-384).  H is
 * symmetric, so the reference's column j equals row j of H; entry (r, c) is
 * evaluated once per unordered pair with dx = x[max(r,c)] - x[min(r,c)] as the
 * reference does (its rows r < c are copies from column r).  Each column is
 * scanned in ascending row order with the point-defect seed at the diagonal,
 * which is the reference's summation order for the diagonal. */
static int calc_jacobian(orc_sim *s, double h, const double *xs)
{
    int n = s->n;
    double c = s->cutoff, c2 = s->cutoff_sqr;
    /* pairwise pass: count then fill an upper-triangle list */
    long cnt = 0;
    int *deg = (int *)calloc((size_t)n, sizeof(int));
    long ucap = 1024;
    int *ui = (int *)malloc(sizeof(int) * ucap), *uj = (int *)malloc(sizeof(int) * ucap);
    double *uv = (double *)malloc(sizeof(double) * ucap);
    for (int j = 0; j < n; ++j)
        for (int i = j + 1; i < n; ++i) {
            double dx = xs[i] - xs[j];
            normalize(&dx);
            double dy = s->y[i] - s->y[j];
            normalize(&dy);
            if (pow(sqrt(dx * dx + dy * dy) - c, 2) < 36.8 * c2) {
                double m = 1;
                if (dx * dx + dy * dy > c2) m = exp(-pow(sqrt(dx * dx + dy * dy) - c, 2) * s->one_per_cutoff_sqr);
                double v = h * s->b[i] * s->b[j] * orc_xy_diff_x(dx, dy) * m;
                if (cnt == ucap) {
                    ucap *= 2;
                    ui = (int *)realloc(ui, sizeof(int) * ucap);
                    uj = (int *)realloc(uj, sizeof(int) * ucap);
                    uv = (double *)realloc(uv, sizeof(double) * ucap);
                }
                ui[cnt] = i;
                uj[cnt] = j;
                uv[cnt] = v;
                cnt++;
                /* an exactly zero value is not copied to the upper part
                 * (getElement treats 0.0 as absent, simulation.cpp:195-229) */
                deg[i] += (v != 0.0);
                deg[j] += 1;
            }
        }
    long nnz = cnt * 2 + n;
    if (nnz > s->cap) {
        free(s->Ai);
        free(s->Ax);
        s->cap = nnz;
        s->Ai = (int *)malloc(sizeof(int) * nnz);
        s->Ax = (double *)malloc(sizeof(double) * nnz);
    }
    /* column pointers: entries above the diagonal (copied, nonzero only), the
     * diagonal, entries below */
    s->Ap[0] = 0;
    for (int j = 0; j < n; ++j) s->Ap[j + 1] = s->Ap[j] + deg[j] + 1;
    int *fill = (int *)malloc(sizeof(int) * n);
    int *diagpos = (int *)malloc(sizeof(int) * n);
    /* rows i<j of column j come from pairs (j, i) with i<j; count them per
     * column first to place the diagonal */
    int *upcnt = (int *)calloc((size_t)n, sizeof(int));
    for (long t = 0; t < cnt; ++t)
        if (uv[t] != 0.0) upcnt[ui[t]]++;
    for (int j = 0; j < n; ++j) {
        diagpos[j] = s->Ap[j] + upcnt[j];
        fill[j] = s->Ap[j];
    }
    /* pairs are enumerated with j (column) ascending, i ascending: rows below
     * the diagonal of column j arrive in order; rows above the diagonal of
     * column i (= row j's) arrive with j ascending too */
    int *lowfill = (int *)malloc(sizeof(int) * n);
    for (int j = 0; j < n; ++j) lowfill[j] = diagpos[j] + 1;
    for (long t = 0; t < cnt; ++t) {
        int i = ui[t], j = uj[t];
        s->Ai[lowfill[j]] = i;
        s->Ax[lowfill[j]++] = uv[t];
        if (uv[t] != 0.0) {
            s->Ai[fill[i]] = j;
            s->Ax[fill[i]++] = uv[t];
        }
    }
    /* diagonal seed from point defects (simulation.cpp:269-325) */
    for (int j = 0; j < n; ++j) {
        double tmp = 0;
        for (int l = 0; l < s->p; ++l) {
            double dx = xs[j] - s->pdx[l];
            normalize(&dx);
            double dy = s->y[j] - s->pdy[l];
            normalize(&dy);
            if (pow(sqrt(dx * dx + dy * dy) - c, 2) < 36.8 * c2) {
                double m = 1;
                if (dx * dx + dy * dy > c2) m = exp(-pow(sqrt(dx * dx + dy * dy) - c, 2) * s->one_per_cutoff_sqr);
                tmp -= s->b[j] * pd_force_dx(dx, dy, s->A, s->KASQR) * m;
            }
        }
        s->Ai[diagpos[j]] = j;
        s->Ax[diagpos[j]] = -tmp * h;
    }
    /* simulation.cpp:349-383: diagonal = -column sum, d, row scaling, +1 */
    for (int j = 0; j < n; ++j) {
        double sub = 0;
        for (int p = s->Ap[j]; p < s->Ap[j + 1]; ++p) sub += s->Ax[p];
        sub *= -1.;
        s->Ax[diagpos[j]] = sub;
        if (sub > 0) {
            sub = 1. / sub;
            sub += 1.;
            sub *= sub;
            s->dvec[j] = 1. / sub;
        } else {
            s->dvec[j] = 0.;
        }
    }
    for (int j = 0; j < n; ++j) {
        for (int p = s->Ap[j]; p < s->Ap[j + 1]; ++p) s->Ax[p] *= (1.0 + s->dvec[s->Ai[p]]) * 0.5;
        s->Ax[diagpos[j]] += 1.0;
    }
    free(deg);
    free(ui);
    free(uj);
    free(uv);
    free(fill);
    free(diagpos);
    free(upcnt);
    free(lowfill);
    return 0;
}

/* simulation.cpp:386-396 */
static void factor(orc_sim *s)
{
    void *sym = NULL;
    (void)umfpack_di_symbolic(s->n, s->n, s->Ap, s->Ai, s->Ax, &sym, NULL, NULL);
    (void)umfpack_di_numeric(s->Ap, s->Ai, s->Ax, sym, &s->numeric, NULL, NULL);
    umfpack_di_free_symbolic(&sym);
}

static void solve(orc_sim *s)
{
    (void)umfpack_di_solve(UMFPACK_A, s->Ap, s->Ai, s->Ax, s->sol, s->g, s->numeric, NULL, NULL);
}

/* Simulation::calculateG, simulation.cpp:133-193 */
static void calc_g(orc_sim *s, double h, double *xn, const double *xo, int use2, int init_speed,
                   int use_init_first, int origin, int end)
{
    double *isp = use2 ? s->v0b : s->v0;
    double *csp = use2 ? s->vs2 : s->vs;
    if (init_speed) {
        double t = s->sim_time, tasi = s->strain;
        if (origin == ST_END_FIRST) {
            t += s->step_size * 0.5;
            tasi += strain_inc(s, s->x, s->x1);
        }
        stress_calc(s, t, origin, tasi);
        s->cur_stress = origin;
        calc_speeds(s, xo, isp, 0);
    }
    if (use_init_first) {
        csp = isp;
    } else {
        double t = s->sim_time + s->step_size, tasi = s->strain;
        if (end == ST_END_FIRST) {
            t -= s->step_size * 0.5;
            tasi += strain_inc(s, s->x, s->x1);
        } else if (end == ST_END_SECOND) {
            tasi += strain_inc(s, s->x, s->x1) + strain_inc(s, s->x1, s->x2);
        } else if (end == ST_END_BIG) {
            tasi += strain_inc(s, s->x, s->xb);
        }
        stress_calc(s, t, end, tasi);
        s->cur_stress = end;
        calc_speeds(s, xn, csp, 0);
    }
    for (int i = 0; i < s->n; ++i)
        s->g[i] = xn[i] - (1.0 + s->dvec[i]) * 0.5 * h * csp[i] - xo[i] - (1.0 - s->dvec[i]) * 0.5 * h * isp[i];
}

/* Simulation::integrate, simulation.cpp:62-84 */
static void integrate(orc_sim *s, double h, double *xn, const double *xo, int use2, int init_speed, int origin,
                      int end)
{
    calc_jacobian(s, h, xn);
    factor(s);
    for (int i = 0; i < s->ic; ++i) {
        if (i > 0) calc_g(s, h, xn, xo, use2, 0, 0, origin, end);
        else calc_g(s, h, xn, xo, use2, init_speed, zero_stress(s), origin, end);
        solve(s);
        for (int j = 0; j < s->n; ++j) xn[j] -= s->sol[j];
    }
    umfpack_di_free_numeric(&s->numeric);
}

static double sum_abs(const double *v, int n)
{
    double a = 0.0;
    for (int i = 0; i < n; ++i) a = a + fabs(v[i]);
    return a;
}

static double sum_sq(const double *v, int n)
{
    double a = 0.0;
    for (int i = 0; i < n; ++i) a = a + v[i] * v[i];
    return a;
}

/* simulation.cpp:443-492 */
static void stage1(orc_sim *s)
{
    s->energy_accum = 0;
    s->vsquare = 0;
    s->cur_stress = ST_ORIGINAL;
    if (s->first_step) {
        stress_calc(s, s->sim_time, ST_ORIGINAL, s->strain);
        calc_speeds(s, s->x, s->v0, 0);
        s->init_speed_needed = 0;
        s->vsquare = sum_sq(s->v0, s->n);
        s->first_step = 0;
    }
    memcpy(s->xb, s->x, sizeof(double) * s->n);
    integrate(s, s->step_size, s->xb, s->x, 0, s->init_speed_needed, ST_ORIGINAL, ST_END_BIG);
    s->successful_step = 0;
}

/* simulation.cpp:494-499 */
static void stage2(orc_sim *s)
{
    memcpy(s->x1, s->x, sizeof(double) * s->n);
    integrate(s, 0.5 * s->step_size, s->x1, s->x, 0, 0, ST_ORIGINAL, ST_END_FIRST);
}

/* simulation.cpp:501-650 (logging, limits and sub-configuration output are
 * host bookkeeping and not restated) */
static void stage3(orc_sim *s)
{
    int n = s->n;
    s->sum_avg_speed = 0;
    memcpy(s->x2, s->x1, sizeof(double) * n);
    integrate(s, 0.5 * s->step_size, s->x2, s->x1, 1, 1, ST_END_FIRST, ST_END_SECOND);
    s->vsquare1 = sum_sq(s->v0, n);
    s->vsquare2 = sum_sq(s->v0b, n);
    s->energy_accum = (s->vsquare1 + s->vsquare2) * 0.5 * s->step_size * 0.5;
    for (int i = 0; i < n; ++i) ph_update_err(s, fabs(s->xb[i] - s->x2[i]), i);
    if (s->max_ratio < 1.0) {
        s->successful_step = 1;
        s->init_speed_needed = 1;
        if (s->calc_strain) {
            s->strain += strain_inc(s, s->x, s->x1);
            s->strain += strain_inc(s, s->x1, s->x2);
        }
        double *t = s->x;
        s->x = s->x2;
        s->x2 = t;
        s->sim_time += s->step_size;
        s->succ++;
        s->cur_stress = ST_ORIGINAL;
        stress_calc(s, s->sim_time, ST_ORIGINAL, s->strain);
        calc_speeds(s, s->x, s->v0, 0);
        s->init_speed_needed = 0;
        s->sum_avg_speed = sum_abs(s->v0, n) / (double)n;
        s->vsquare = sum_sq(s->v0, n);
        s->energy_accum += (s->vsquare2 + s->vsquare) * 0.5 * s->step_size * 0.5;
        s->energy += s->energy_accum;
    } else {
        s->failed++;
    }
    s->step_size = ph_new_step(s, s->step_size);
    s->last_ratio = s->max_ratio;
    memcpy(s->last_tol, s->tol, sizeof(double) * n);
    ph_reset(s);
    if (s->max_step_limited && s->max_step < s->step_size) s->step_size = s->max_step;
}

/* ------------------------------------------------------------ exports --- */

void *ref_create(int n, const double *xyb, int p, const double *pd, const ref_params *prm)
{
    orc_sim *s = (orc_sim *)calloc(1, sizeof(orc_sim));
    s->n = n;
    s->p = p;
    s->x = dalloc(n);
    s->y = dalloc(n);
    s->b = dalloc(n);
    s->xb = dalloc(n);
    s->x1 = dalloc(n);
    s->x2 = dalloc(n);
    s->pdx = dalloc(p);
    s->pdy = dalloc(p);
    s->v0 = dalloc(n);
    s->v0b = dalloc(n);
    s->vs = dalloc(n);
    s->vs2 = dalloc(n);
    s->g = dalloc(n);
    s->dvec = dalloc(n);
    s->sol = dalloc(n);
    s->tol = dalloc(n);
    s->errv = dalloc(n);
    s->last_tol = dalloc(n);
    for (int i = 0; i < n; ++i) {
        s->x[i] = xyb[3 * i];
        s->y[i] = xyb[3 * i + 1];
        s->b[i] = xyb[3 * i + 2];
    }
    for (int i = 0; i < p; ++i) {
        s->pdx[i] = pd[2 * i];
        s->pdy[i] = pd[2 * i + 1];
    }
    /* SimulationData() defaults (simulation_data.cpp:43-109, constants.h) */
    s->A = 1e-4 * 16.0;
    s->KASQR = 1.65 * 1.65 * 1e6 / 256.0;
    s->ic = 2;
    s->cutoff_multiplier = 1.0;
    update_cutoff(s);
    /* processInput (project_parser.cpp:174-212) */
    s->step_size = prm->step_size;
    s->prec = prm->prec;
    s->cutoff_multiplier = prm->cutoff_multiplier;
    update_cutoff(s);
    s->max_step_limited = prm->max_step_limited;
    s->max_step = prm->max_step;
    if (prm->pd_scaling) {
        s->A *= 1. / sqrt((double)n);
        s->KASQR *= (double)n;
    }
    s->calc_strain = prm->calculate_strain;
    s->order_param = prm->order_parameter;
    s->stress_kind = prm->stress_kind;
    s->stress_rate = prm->stress_rate;
    s->spring_k = prm->spring_constant;
    s->stress_value = prm->stress_value;
    /* Simulation::Simulation (simulation.cpp:38-55): PrecisionHandler with the
     * precision set (setMinPrecisity) and sized to N */
    s->prec_sqr = s->prec * s->prec;
    ph_reset(s);
    s->first_step = 1;
    s->init_speed_needed = 1;
    s->successful_step = 1;
    s->Ap = (int *)calloc((size_t)n + 1, sizeof(int));
    return s;
}

void ref_destroy(void *hp)
{
    orc_sim *s = (orc_sim *)hp;
    if (!s) return;
    double *bufs[] = {s->x, s->y, s->b, s->xb, s->x1, s->x2, s->pdx, s->pdy, s->v0, s->v0b, s->vs,
                      s->vs2, s->g, s->dvec, s->sol, s->tol, s->errv, s->last_tol, s->Ax};
    for (size_t i = 0; i < sizeof(bufs) / sizeof(bufs[0]); ++i) free(bufs[i]);
    free(s->Ap);
    free(s->Ai);
    if (s->numeric) umfpack_di_free_numeric(&s->numeric);
    free(s);
}

void ref_get_params(void *hp, double *out)
{
    orc_sim *s = (orc_sim *)hp;
    out[0] = s->cutoff;
    out[1] = s->cutoff_sqr;
    out[2] = s->one_per_cutoff_sqr;
    out[3] = s->A;
    out[4] = s->KASQR;
    out[5] = s->prec;
    out[6] = s->step_size;
    out[7] = s->ic;
}

int ref_step(void *hp)
{
    orc_sim *s = (orc_sim *)hp;
    stage1(s);
    stage2(s);
    stage3(s);
    return s->successful_step;
}

void ref_get_scalars(void *hp, double *out)
{
    orc_sim *s = (orc_sim *)hp;
    out[0] = s->sim_time;
    out[1] = s->step_size;
    out[2] = (double)s->succ;
    out[3] = (double)s->failed;
    out[4] = s->energy;
    out[5] = s->strain;
    out[6] = s->last_ratio;
    out[7] = s->sum_avg_speed;
    out[8] = s->vsquare;
    out[9] = s->energy_accum;
    out[10] = s->cutoff;
    out[11] = stress_get(s, ST_ORIGINAL);
}

void ref_get_config(void *hp, int which, double *xyb)
{
    orc_sim *s = (orc_sim *)hp;
    const double *x = s->x;
    if (which == 1) x = s->xb;
    if (which == 2) x = s->x1;
    if (which == 3) x = s->x2;
    for (int i = 0; i < s->n; ++i) {
        xyb[3 * i] = x[i];
        xyb[3 * i + 1] = s->y[i];
        xyb[3 * i + 2] = s->b[i];
    }
}

void ref_get_vector(void *hp, int which, double *out)
{
    orc_sim *s = (orc_sim *)hp;
    const double *v = s->v0;
    if (which == 1) v = s->v0b;
    if (which == 2) v = s->vs;
    if (which == 3) v = s->vs2;
    if (which == 4) v = s->dvec;
    if (which == 5) v = s->g;
    if (which == 6) v = s->last_tol;
    memcpy(out, v, sizeof(double) * s->n);
}

void ref_set_state(void *hp, const double *xyb, double step_size, double sim_time, double energy,
                   double strain, int first_step)
{
    orc_sim *s = (orc_sim *)hp;
    for (int i = 0; i < s->n; ++i) {
        s->x[i] = xyb[3 * i];
        s->y[i] = xyb[3 * i + 1];
        s->b[i] = xyb[3 * i + 2];
    }
    s->step_size = step_size;
    s->sim_time = sim_time;
    s->strain = strain;
    s->energy = energy;
    ph_reset(s);
    if (first_step) {
        s->first_step = 1;
        s->init_speed_needed = 1;
        return;
    }
    s->first_step = 0;
    s->cur_stress = ST_ORIGINAL;
    stress_calc(s, s->sim_time, ST_ORIGINAL, s->strain);
    calc_speeds(s, s->x, s->v0, 0);
    s->init_speed_needed = 0;
    ph_reset(s);
}

void ref_speeds(void *hp, const double *xyb, double sim_time, int stress_type, double *v, double *tol)
{
    orc_sim *s = (orc_sim *)hp;
    double *xs = dalloc(s->n);
    double *ys = s->y, *bs = s->b;
    double *ty = dalloc(s->n), *tb = dalloc(s->n);
    for (int i = 0; i < s->n; ++i) {
        xs[i] = xyb[3 * i];
        ty[i] = xyb[3 * i + 1];
        tb[i] = xyb[3 * i + 2];
    }
    s->y = ty;
    s->b = tb;
    stress_calc(s, sim_time, stress_type, s->strain);
    s->cur_stress = stress_type;
    ph_reset(s);
    calc_speeds(s, xs, v, 0);
    memcpy(tol, s->tol, sizeof(double) * s->n);
    ph_reset(s);
    s->y = ys;
    s->b = bs;
    free(xs);
    free(ty);
    free(tb);
}

long ref_jacobian(void *hp, double stepsize, const double *xyb, int *Ap, int *Ai, double *Ax, double *dvec,
                  long cap)
{
    orc_sim *s = (orc_sim *)hp;
    double *xs = dalloc(s->n);
    double *ys = s->y, *bs = s->b;
    double *ty = dalloc(s->n), *tb = dalloc(s->n);
    for (int i = 0; i < s->n; ++i) {
        xs[i] = xyb[3 * i];
        ty[i] = xyb[3 * i + 1];
        tb[i] = xyb[3 * i + 2];
    }
    s->y = ty;
    s->b = tb;
    calc_jacobian(s, stepsize, xs);
    s->y = ys;
    s->b = bs;
    free(xs);
    free(ty);
    free(tb);
    long nnz = s->Ap[s->n];
    if (nnz > cap) return -nnz;
    memcpy(Ap, s->Ap, sizeof(int) * (s->n + 1));
    memcpy(Ai, s->Ai, sizeof(int) * nnz);
    memcpy(Ax, s->Ax, sizeof(double) * nnz);
    memcpy(dvec, s->dvec, sizeof(double) * s->n);
    return nnz;
}

void ref_integrate_stage(void *hp, int stage, double *x_out)
{
    orc_sim *s = (orc_sim *)hp;
    if (stage == 1) {
        memcpy(s->xb, s->x, sizeof(double) * s->n);
        integrate(s, s->step_size, s->xb, s->x, 0, s->init_speed_needed, ST_ORIGINAL, ST_END_BIG);
        memcpy(x_out, s->xb, sizeof(double) * s->n);
    } else if (stage == 2) {
        memcpy(s->x1, s->x, sizeof(double) * s->n);
        integrate(s, 0.5 * s->step_size, s->x1, s->x, 0, 0, ST_ORIGINAL, ST_END_FIRST);
        memcpy(x_out, s->x1, sizeof(double) * s->n);
    } else {
        memcpy(s->x2, s->x1, sizeof(double) * s->n);
        integrate(s, 0.5 * s->step_size, s->x2, s->x1, 1, 1, ST_END_FIRST, ST_END_SECOND);
        memcpy(x_out, s->x2, sizeof(double) * s->n);
    }
}

void ref_field(int which, long n, const double *dx, const double *dy, double *out)
{
    for (long i = 0; i < n; ++i)
        out[i] = which == 0 ? orc_xy(dx[i], dy[i]) : which == 1 ? orc_xy_diff_x(dx[i], dy[i]) : orc_xy_diff_x2(dx[i], dy[i]);
}

/* ------------------------------------------------ eigenvalue analysis --- */
/* The --ev-analyzation mode: SpectralDecompositor::decompose
 * (spectral_decompositor.cpp:63-165) builds the dense Hessian of the
 * configuration; TimeSeriesProcessor (time_series_processor.cpp:21-247)
 * derives its observables from the eigenpairs.  The eigensolver itself is
 * LAPACKE_dsyevd (spectral_decompositor.cpp:188); the Python side of the
 * oracle uses numpy.linalg.eigh, which calls the same LAPACK driver. */

/* AnalyticField.cpp:95-108: d2/dx2 of fpair (no Taylor branch) */
static double fpair_dx2(double dx, double cos2piy, double dy)
{
    double ch = cosh(M_PI * 2.0 * dx);
    double sh = sinh(M_PI * 2.0 * dx);
    double c4y = cos(4.0 * M_PI * dy);
    double ch4 = cosh(M_PI * 4.0 * dx);
    double sh4 = sinh(M_PI * 4.0 * dx);
    return (4.0 * M_PI *
            (sh * cos2piy * (pow(cos2piy, 2.0) - 2.0) + 2.0 * M_PI * dx * pow(sh, 2.0) * (c4y - 2.0) -
             M_PI * dx * pow(ch, 3.0) * cos2piy + 0.5 * M_PI * dx * ch * cos2piy * (2.0 * ch4 + c4y - 5.0) +
             pow(ch, 2.0) * (2.0 * M_PI * dx - sh * cos2piy) + sh4)) /
           pow(cos2piy - ch, 4.0);
}

/* AnalyticField.cpp:122-132 */
static double gimg_dx2(int images, double dx, double cos2piy, double dy)
{
    double s = fpair_dx2(dx, cos2piy, dy);
    for (int k = 1; k <= images; ++k)
        s = s + fpair_dx2(dx - (double)k, cos2piy, dy) + fpair_dx2(dx + (double)k, cos2piy, dy);
    return s;
}

/* AnalyticField::xy_diff_x2, AnalyticField.cpp:183-202 */
double orc_xy_diff_x2(double dx, double dy)
{
    const double n = (double)ORC_FIELD_N;
    double cy = cos(M_PI * 2.0 * dy);
    if (dx < 0)
        return -2.0 * fpair_dx(dx + n + 1.0, cy, dy) - dx * fpair_dx2(dx + n + 1.0, cy, dy) +
               fpair_dx2(dx - n, cy, dy) * (1.0 + dx) + 2.0 * fpair_dx(dx - n, cy, dy) + fpair_dx2(dx + n, cy, dy) +
               gimg_dx2(ORC_FIELD_N - 1, dx, cy, dy);
    return 2.0 * fpair_dx(dx - n - 1.0, cy, dy) + dx * fpair_dx2(dx - n - 1.0, cy, dy) +
           fpair_dx2(dx + n, cy, dy) * (1.0 - dx) - 2.0 * fpair_dx(dx + n, cy, dy) + fpair_dx2(dx - n, cy, dy) +
           gimg_dx2(ORC_FIELD_N - 1, dx, cy, dy);
}

/* spectral_decompositor.cpp:63-165: H (row-major n x n) with
 * H_ij = b_i b_j xy_diff_x(x_i - x_j, y_i - y_j) for i != j and
 * H_ii = -sum_{j<i} H_ij - sum_defects b_i d/dx(defect force) - sum_{j>i} H_ji,
 * accumulated in that order.  The defects use their own scaling: A = 1.6e-3 /
 * sqrt(defect count), K = 1.65^2 1e6 / 256 * n (:76-84). */
void orc_ev_hessian(int n, const double *xyb, int p, const double *pd, double *H)
{
    double sdA = 0.0, sdK = 0.0;
    if (p > 0) {
        sdA = 1e-4 * 16.0 * 1. / sqrt((double)p);
        sdK = 1.65 * 1.65 * 1e6 / 256.0 * (double)n;
    }
    memset(H, 0, sizeof(double) * (size_t)n * (size_t)n);
    for (int i = 0; i < n; ++i) {
        double sub = 0.0;
        for (int j = 0; j < i; ++j) {
            double dx = xyb[3 * i] - xyb[3 * j];
            normalize(&dx);
            double dy = xyb[3 * i + 1] - xyb[3 * j + 1];
            normalize(&dy);
            double t = xyb[3 * i + 2] * xyb[3 * j + 2] * orc_xy_diff_x(dx, dy);
            sub += t;
            H[(size_t)i * n + j] = t;
            H[(size_t)j * n + i] = t;
        }
        H[(size_t)i * n + i] -= sub;
        for (int k = 0; k < p; ++k) {
            double dx = xyb[3 * i] - pd[2 * k];
            normalize(&dx);
            double dy = xyb[3 * i + 1] - pd[2 * k + 1];
            normalize(&dy);
            H[(size_t)i * n + i] -= xyb[3 * i + 2] * pd_force_dx(dx, dy, sdA, sdK);
        }
    }
    for (int i = 0; i < n; ++i)
        for (int j = i + 1; j < n; ++j) H[(size_t)i * n + i] -= H[(size_t)j * n + i];
}

/* TimeSeriesProcessor::calculateHessianDerivative (time_series_processor.cpp:208-247) */
static double ev_hess_deriv(int n, const double *xyb, int i, int j, int k)
{
    double dx, dy;
    if (i == j && j == k) {
        double sum = 0.0;
        for (int l = 0; l < n; ++l) {
            if (l == i) continue;
            dx = xyb[3 * i] - xyb[3 * l];
            dy = xyb[3 * i + 1] - xyb[3 * l + 1];
            normalize(&dx);
            normalize(&dy);
            sum += xyb[3 * l + 2] * orc_xy_diff_x2(dx, dy);
        }
        return -xyb[3 * i + 2] * sum;
    }
    if (i == j || i == k) {
        const int o = i == j ? k : j;
        dx = xyb[3 * i] - xyb[3 * o];
        dy = xyb[3 * i + 1] - xyb[3 * o + 1];
        normalize(&dx);
        normalize(&dy);
        return xyb[3 * i + 2] * xyb[3 * o + 2] * orc_xy_diff_x2(dx, dy);
    }
    if (j == k) {
        dx = xyb[3 * i] - xyb[3 * j];
        dy = xyb[3 * i + 1] - xyb[3 * j + 1];
        normalize(&dx);
        normalize(&dy);
        return -xyb[3 * i + 2] * xyb[3 * j + 2] * orc_xy_diff_x2(dx, dy);
    }
    return 0.0;
}

/* The eigenvalue derivatives, literally as time_series_processor.cpp:104-121
 * loops them (n^4 terms; small n only): V holds eigenvector m at V[m n ..],
 * speeds the velocities at the configuration, sderiv the stress protocol's
 * getStressDerivative. */
void orc_ev_deriv_literal(int n, const double *xyb, const double *V, const double *speeds, double sderiv,
                          double *out)
{
    for (int m = 0; m < n; ++m) {
        double sum = 0.0;
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) {
                double mult = V[(size_t)m * n + i] * V[(size_t)m * n + j] / sderiv;
                double sub = 0.0;
                for (int k = 0; k < n; ++k) sub += speeds[k] * ev_hess_deriv(n, xyb, i, j, k);
                sum += sub * mult;
            }
        out[m] = sum;
    }
}

/* The correlation matrices of time_series_processor.cpp:145-197: for every
 * mode m three S x S histograms over the ordered pairs i != j, binned by
 * (floor((dx + 1/2) S), floor((dy + 1/2) S)) of the minimum-image
 * separation and weighted by V_mj^2 V_mi^2: equal signs (pp), opposite signs
 * (pn), all pairs (pppn).  out: [m][pp, pn, pppn][S][S]. */
void orc_ev_correl_literal(int n, const double *xyb, const double *V, int S, double *out)
{
    const size_t ss = (size_t)S * S;
    memset(out, 0, sizeof(double) * (size_t)n * 3 * ss);
    for (int m = 0; m < n; ++m) {
        double *pp = out + (size_t)m * 3 * ss, *pn = pp + ss, *pppn = pn + ss;
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) {
                if (i == j) continue;
                double dx = xyb[3 * i] - xyb[3 * j];
                double dy = xyb[3 * i + 1] - xyb[3 * j + 1];
                normalize(&dx);
                normalize(&dy);
                int tx = (int)floor((dx + 0.5) * S);
                int ty = (int)floor((dy + 0.5) * S);
                double w = pow(V[(size_t)m * n + j], 2.0) * pow(V[(size_t)m * n + i], 2.0);
                if (xyb[3 * i + 2] != xyb[3 * j + 2]) pn[(size_t)tx * S + ty] += w;
                if (xyb[3 * i + 2] == xyb[3 * j + 2]) pp[(size_t)tx * S + ty] += w;
                pppn[(size_t)tx * S + ty] += w;
            }
    }
}
