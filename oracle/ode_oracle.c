/*
 * ode_oracle.c - CPU oracle for odesolve_2D sweeps (FP64, one point after another).
 *
 * Oracle infrastructure only (tests/, smoke, the bench CPU leg); built by gcc into
 * oracle/_build/libode_oracle.so. It restates, for a hand-written right-hand side, the
 * integrators of the sweep path:
 *
 *   method 0  classical RK4 with the reference step structure (gqis/cuda_solvers.py:470-517):
 *             stage times t + dt/2 and (t + dt/2) + dt/2 from the step index, k1 reused from
 *             the end of the previous step;
 *   method 1  adaptive Tsit5 between uniform output times (gqis/cuda_solvers.py:731-908):
 *             RMS error norm, factor 0.9 err^-1/5 limited to [0.2, 5], the step that reaches
 *             the output time shortened to end on it, h kept across intervals, more than
 *             max_substeps attempts per interval -> NaN;
 *   method 2  adaptive DOP853 (Hairer, Norsett & Wanner): 5th/3rd-order combined error
 *             err5^2 / sqrt(err5^2 + 0.01 err3^2) * h / sqrt(n), factor 0.9 err^-1/8 limited
 *             to [0.2, 10], no growth right after a rejection, same output-interval rules.
 *
 * Tableaus are passed in by the caller (oracle/ode_oracle.py). Models:
 *   0  Duffing  x' = v, v' = -gamma v - x - beta x^3 + F cos(W t);  p = {gamma, beta, F, W}
 *   1  x' = -x, y' = t                                                (analytic test)
 * Outputs per point: final state, the state at every output time (trace, optional),
 * accepted / rejected step counts.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define MAXS 16
#define MAXN 4

static void model_rhs(int model, double t, const double* y, double* dy, const double* p) {
    if (model == 0) {
        dy[0] = y[1];
        dy[1] = -p[0] * y[1] - y[0] - p[1] * y[0] * y[0] * y[0] + p[2] * cos(p[3] * t);
    } else {
        dy[0] = -y[0];
        dy[1] = t;
    }
}

typedef struct {
    int ns;
    const double* c;   /* [ns] */
    const double* a;   /* [ns * ns] row-major */
    const double* b;   /* [ns] */
    const double* e;   /* tsit5: [ns + 1] (last weights f(y_new)); dop853: e5 [ns] */
    const double* e3;  /* dop853: [ns] */
} tableau;

static void rk4_point(int model, int n, const double* p, const double* y0, double t_in, double dt,
                      int nsteps, double* final_state, double* trace) {
    double y[MAXN], k[MAXN], yt[MAXN], acc[MAXN];
    memcpy(y, y0, sizeof(double) * n);
    const double h2 = dt * 0.5, h6 = dt / 6.0;
    model_rhs(model, t_in + 0.0, y, k, p);
    for (int step = 0; step < nsteps; ++step) {
        double tm = ((double)step + 0.5) * dt;
        for (int i = 0; i < n; ++i) { yt[i] = fma(h2, k[i], y[i]); acc[i] = k[i]; }
        model_rhs(model, t_in + tm, yt, k, p);
        for (int i = 0; i < n; ++i) { yt[i] = fma(h2, k[i], y[i]); acc[i] = fma(2.0, k[i], acc[i]); }
        model_rhs(model, t_in + tm, yt, k, p);
        tm += h2;
        for (int i = 0; i < n; ++i) { yt[i] = fma(dt, k[i], y[i]); acc[i] = fma(2.0, k[i], acc[i]); }
        model_rhs(model, t_in + tm, yt, k, p);
        for (int i = 0; i < n; ++i) { acc[i] += k[i]; y[i] = fma(h6, acc[i], y[i]); }
        if (step + 1 < nsteps) model_rhs(model, t_in + tm, y, k, p);
        if (trace) memcpy(trace + (size_t)step * n, y, sizeof(double) * n);
    }
    memcpy(final_state, y, sizeof(double) * n);
}

/* One attempt of an embedded pair; returns the error norm, writes y_new and f(t+h, y_new). */
static double attempt(int method, int model, int n, const double* p, const tableau* T, double t, double h,
                      const double* y, const double* k1, double* y_new, double* k_next,
                      double rtol, double atol) {
    double k[MAXS][MAXN], yt[MAXN];
    const int ns = T->ns;
    memcpy(k[0], k1, sizeof(double) * n);
    for (int s = 1; s < ns; ++s) {
        for (int i = 0; i < n; ++i) {
            double acc = 0.0;
            for (int j = 0; j < s; ++j) acc += T->a[s * ns + j] * k[j][i];
            yt[i] = y[i] + h * acc;
        }
        model_rhs(model, t + T->c[s] * h, yt, k[s], p);
    }
    for (int i = 0; i < n; ++i) {
        double acc = 0.0;
        for (int j = 0; j < ns; ++j) acc += T->b[j] * k[j][i];
        y_new[i] = y[i] + h * acc;
    }
    model_rhs(model, t + h, y_new, k_next, p);
    if (method == 1) {
        double sum = 0.0;
        for (int i = 0; i < n; ++i) {
            double e = T->e[ns] * k_next[i];
            for (int j = 0; j < ns; ++j) e += T->e[j] * k[j][i];
            e *= h;
            const double sc = rtol * fmax(fabs(y[i]), fabs(y_new[i])) + atol;
            sum += (e / sc) * (e / sc);
        }
        return sqrt(sum / n);
    }
    double e5 = 0.0, e3 = 0.0;
    for (int i = 0; i < n; ++i) {
        double x5 = 0.0, x3 = 0.0;
        for (int j = 0; j < ns; ++j) { x5 += T->e[j] * k[j][i]; x3 += T->e3[j] * k[j][i]; }
        const double sc = rtol * fmax(fabs(y[i]), fabs(y_new[i])) + atol;
        x5 /= sc;
        x3 /= sc;
        e5 += x5 * x5;
        e3 += x3 * x3;
    }
    if (e5 == 0.0 && e3 == 0.0) return 0.0;
    return fabs(h) * e5 / sqrt((e5 + 0.01 * e3) * n);
}

static void adaptive_point(int method, int model, int n, const double* p, const tableau* T, const double* y0,
                           double t_in, double dt, int nsteps, double rtol, double atol, int max_substeps,
                           double* final_state, double* trace, int* counts) {
    double y[MAXN], k1[MAXN], y_new[MAXN], k_next[MAXN];
    const double expo = method == 1 ? -0.2 : -1.0 / 8.0;
    const double fmax_ = method == 1 ? 5.0 : 10.0;
    memcpy(y, y0, sizeof(double) * n);
    model_rhs(model, t_in, y, k1, p);
    double h = dt;
    int accepted = 0, rejected = 0, failed = 0, rejected_last = 0;
    for (int step = 0; step < nsteps && !failed; ++step) {
        double tau = 0.0;
        int substeps = 0;
        while (tau < dt) {
            const double remaining = dt - tau;
            const int last = h * 1.01 >= remaining;
            const double hs = last ? remaining : h;
            const double t = t_in + ((double)step * dt + tau);
            const double err = attempt(method, model, n, p, T, t, hs, y, k1, y_new, k_next, rtol, atol);
            double factor = 0.9 * pow(err, expo);
            factor = fmin(fmax_, fmax(0.2, factor));
            if (err <= 1.0) {
                ++accepted;
                if (method == 2 && rejected_last) factor = fmin(1.0, factor);
                rejected_last = 0;
                memcpy(y, y_new, sizeof(double) * n);
                memcpy(k1, k_next, sizeof(double) * n);
                tau = last ? dt : tau + hs;
                h = last ? fmax(h, hs * factor) : hs * factor;
            } else {
                ++rejected;
                rejected_last = 1;
                h = hs * factor;
            }
            if (++substeps > max_substeps) {
                failed = 1;
                for (int i = 0; i < n; ++i) y[i] = NAN;
                break;
            }
        }
        if (trace) memcpy(trace + (size_t)step * n, y, sizeof(double) * n);
    }
    memcpy(final_state, y, sizeof(double) * n);
    if (counts) { counts[0] = accepted; counts[1] = rejected; }
}

/* Sweep over npts points: params is [npts * np], y0 is [npts * n]. trace (optional) is
 * [npts * nsteps * n]; counts (optional) is [npts * 2]. Returns 0, or -1 on bad arguments. */
int oracle_sweep(int method, int model, int n, int np, int npts, const double* params, const double* y0,
                 double t_in, double dt, int nsteps, double rtol, double atol, int max_substeps, int ns,
                 const double* c, const double* a, const double* b, const double* e, const double* e3,
                 double* final_state, double* trace, int* counts) {
    if (n < 1 || n > MAXN || ns > MAXS || npts < 0 || nsteps < 1) return -1;
    tableau T = {ns, c, a, b, e, e3};
    for (int q = 0; q < npts; ++q) {
        const double* p = params + (size_t)q * np;
        double* tr = trace ? trace + (size_t)q * nsteps * n : NULL;
        if (method == 0)
            rk4_point(model, n, p, y0 + (size_t)q * n, t_in, dt, nsteps, final_state + (size_t)q * n, tr);
        else
            adaptive_point(method, model, n, p, &T, y0 + (size_t)q * n, t_in, dt, nsteps, rtol, atol, max_substeps,
                           final_state + (size_t)q * n, tr, counts ? counts + 2 * q : NULL);
    }
    return 0;
}
