/*
 * FP64 CPU oracle for the fused Dopri5 + steady-state-feature hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker that the CUDA kernels in
 * pybasin_b200/csrc are compared against (tests/, __graft_entry__.smoke() and
 * the cpu_baseline / reference arm of bench.py).  It is never linked into the
 * product library and the product never calls it.
 *
 * What it restates (reference paths are relative to the pybasin project root):
 *   - Dormand-Prince 5(4) step, tableau, Shampine error coefficients and the
 *     torchdiffeq-style 4th-order dense output:
 *       src/zigode/src/solver/dopri5_generic.zig:16-56  (coefficients)
 *       src/zigode/src/solver/dopri5_generic.zig:77-242 (solve_into main loop)
 *       src/zigode/src/solver/dopri5_generic.zig:185-192 (RMS error norm)
 *       src/zigode/src/solver/dopri5_generic.zig:197-218 (dense output)
 *       src/zigode/src/solver/dopri5_generic.zig:228-235 (step-size control)
 *       src/zigode/src/solver/dopri5_generic.zig:270-321 (initial step size)
 *   - pthread batch over ICs: src/zigode/src/c_api.zig:193-314 (here: OpenMP).
 *   - Right-hand sides: case_studies/pendulum/pendulum_ode.py:23-46,
 *     case_studies/duffing_oscillator/duffing_ode.py:26-42,
 *     case_studies/lorenz/lorenz_ode.py:28-64 (masked variant) and
 *     case_studies/lorenz/lorenz_jax_ode.py (plain variant),
 *     tests/unit/solvers/test_solver.py:16-21 (linear decay).
 *   - Window statistics computed the way the reference's torch calculators do
 *     (two-pass, over the stored samples):
 *       src/pybasin/ts_torch/calculators/torch_features_statistical.py:30-110,307-318
 *       src/pybasin/ts_torch/calculators/torch_features_pattern.py:56-60
 *
 * Extensions over the Zig solver (documented, shared with the CUDA kernels):
 *   - per-trajectory status (ok / max_steps / dt underflow / unbounded / non-finite),
 *   - an optional unbounded threshold that stops a trajectory once max|y| >= thr
 *     after an accepted step (the diffrax Event used by JaxSolver,
 *     src/pybasin/solvers/jax_solver.py:375-436 and
 *     case_studies/lorenz/setup_lorenz_system.py:16-26), after which the
 *     remaining save points are +inf.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "oracle.h"

/* ---- Dormand-Prince tableau (published method constants) ---------------- */
static const double A21 = 1.0 / 5.0;
static const double A31 = 3.0 / 40.0, A32 = 9.0 / 40.0;
static const double A41 = 44.0 / 45.0, A42 = -56.0 / 15.0, A43 = 32.0 / 9.0;
static const double A51 = 19372.0 / 6561.0, A52 = -25360.0 / 2187.0, A53 = 64448.0 / 6561.0,
                    A54 = -212.0 / 729.0;
static const double A61 = 9017.0 / 3168.0, A62 = -355.0 / 33.0, A63 = 46732.0 / 5247.0,
                    A64 = 49.0 / 176.0, A65 = -5103.0 / 18656.0;
static const double B1 = 35.0 / 384.0, B3 = 500.0 / 1113.0, B4 = 125.0 / 192.0,
                    B5 = -2187.0 / 6784.0, B6 = 11.0 / 84.0;
static const double C2 = 1.0 / 5.0, C3 = 3.0 / 10.0, C4 = 4.0 / 5.0, C5 = 8.0 / 9.0;
static const double E1 = 35.0 / 384.0 - 1951.0 / 21600.0;
static const double E3 = 500.0 / 1113.0 - 22642.0 / 50085.0;
static const double E4 = 125.0 / 192.0 - 451.0 / 720.0;
static const double E5 = -2187.0 / 6784.0 - -12231.0 / 42400.0;
static const double E6 = 11.0 / 84.0 - 649.0 / 6300.0;
static const double E7 = -1.0 / 60.0;
static const double M1 = 6025192743.0 / 30085553152.0 / 2.0;
static const double M3 = 51252292925.0 / 65400821598.0 / 2.0;
static const double M4 = -2691868925.0 / 45128329728.0 / 2.0;
static const double M5 = 187940372067.0 / 1594534317056.0 / 2.0;
static const double M6 = -1776094331.0 / 19743644256.0 / 2.0;
static const double M7 = 11237099.0 / 235043384.0 / 2.0;

static const double SAFETY = 0.9, MIN_FACTOR = 0.2, MAX_FACTOR = 10.0;

/* ---- right-hand sides ---------------------------------------------------- */
static void rhs(int sys, double t, const double *y, double *dy, const double *p, int dim,
                const oracle_aux *aux)
{
    switch (sys) {
    case ORACLE_SYS_LINEAR: /* dy/dt = p0 * y (every component) */
        for (int i = 0; i < dim; ++i) dy[i] = p[0] * y[i];
        break;
    case ORACLE_SYS_PENDULUM: /* [alpha, T, K] */
        dy[0] = y[1];
        dy[1] = -p[0] * y[1] + p[1] - p[2] * sin(y[0]);
        break;
    case ORACLE_SYS_DUFFING: /* [delta, k3, A] */
        dy[0] = y[1];
        dy[1] = -p[0] * y[1] - p[1] * y[0] * y[0] * y[0] + p[2] * cos(t);
        break;
    case ORACLE_SYS_LORENZ: /* [sigma, r, b] */
    case ORACLE_SYS_LORENZ_MASKED: {
        double f0 = p[0] * (y[1] - y[0]);
        double f1 = p[1] * y[0] - y[0] * y[2] - y[1];
        double f2 = y[0] * y[1] - p[2] * y[2];
        if (sys == ORACLE_SYS_LORENZ_MASKED) {
            double m = fmax(fabs(y[0]), fmax(fabs(y[1]), fabs(y[2])));
            if (!(m < 200.0)) f0 = f1 = f2 = 0.0;
        }
        dy[0] = f0; dy[1] = f1; dy[2] = f2;
        break;
    }
    case ORACLE_SYS_ROSSLER_NET: { /* [a, b, c, K]; state = [x(0..n), y(0..n), z(0..n)] */
        int n = dim / 3;
        const double *x = y, *yy = y + n, *z = y + 2 * n;
        for (int i = 0; i < n; ++i) {
            double lap = 0.0;
            for (int e = aux->row_ptr[i]; e < aux->row_ptr[i + 1]; ++e) lap += x[aux->col_idx[e]] - x[i];
            dy[i] = -yy[i] - z[i] + p[3] * lap;
            dy[n + i] = x[i] + p[0] * yy[i];
            dy[2 * n + i] = p[1] + z[i] * (x[i] - p[2]);
        }
        break;
    }
    case ORACLE_SYS_FRICTION: { /* [v_d, xi, musd, mud, muv, v0]; case_studies/friction/friction_ode.py:32-75 */
        const double vd = p[0], xi = p[1], musd = p[2], mud = p[3], muv = p[4], v0 = p[5];
        const double disp = y[0], vel = y[1];
        const double vrel = vel - vd, eta = 1e-4, k_smooth = 50.0;
        const double f_fric = mud + mud * (musd - 1.0) * exp(-fabs(vrel) / v0) + muv * fabs(vrel) / v0;
        const int slip = fabs(vrel) > eta;
        const int trans = fabs(disp + 2.0 * xi * vel) > mud * musd;
        const double slip_vel = -disp - 2.0 * xi * vel - tanh(k_smooth * vrel) * f_fric;
        const double trans_vel = -disp - 2.0 * xi * vel + mud * musd * tanh(k_smooth * f_fric);
        const double stick_vel = -(vel - vd);
        dy[0] = (slip || trans) ? vel : vd;
        dy[1] = slip ? slip_vel : (trans ? trans_vel : stick_vel);
        break;
    }
    default:
        for (int i = 0; i < dim; ++i) dy[i] = NAN;
    }
}

/* ---- window statistics (two-pass over stored samples) -------------------- */
static int cmp_double(const void *a, const void *b)
{
    double x = *(const double *)a, y = *(const double *)b;
    return (x > y) - (x < y);
}

/* ascending with every NaN after the numbers (the order of torch.sort) */
static int cmp_double_nan_last(const void *a, const void *b)
{
    double x = *(const double *)a, y = *(const double *)b;
    if (isnan(x) || isnan(y)) return (isnan(x) != 0) - (isnan(y) != 0);
    return (x > y) - (x < y);
}

/* Power |X_k|^2 of the one-sided DFT (rfft, k = 0..n/2) of w - shift, by direct
   sums with the phase k*i reduced exactly modulo n. */
static void power_spectrum(const double *w, int n, double shift, double *psd)
{
    const double two_pi = 6.283185307179586476925286766559;
    for (int k = 0; k <= n / 2; ++k) {
        double re = 0.0, im = 0.0;
        long ph = 0;
        for (int i = 0; i < n; ++i) {
            const double ang = two_pi * (double)ph / n;
            re += (w[i] - shift) * cos(ang);
            im -= (w[i] - shift) * sin(ang);
            ph += k;
            if (ph >= n) ph -= n;
        }
        psd[k] = re * re + im * im;
    }
}

/* torch_features_trend.py:11-51: least squares of a on t = 0..n-1, attribute 0..4
   = slope, intercept, rvalue, the reference's pseudo p-value 1 / (1 + |t|), stderr */
static double trend_attr(const double *a, int n, int attr)
{
    double am = 0.0;
    for (int i = 0; i < n; ++i) am += a[i];
    am /= n;
    const double tm = 0.5 * (n - 1.0);
    double ss_tt = 0.0, ss_tx = 0.0, ss_xx = 0.0;
    for (int i = 0; i < n; ++i) {
        ss_tt += (i - tm) * (i - tm);
        ss_tx += (i - tm) * (a[i] - am);
        ss_xx += (a[i] - am) * (a[i] - am);
    }
    const double slope = ss_tx / (ss_tt + 1e-10), intercept = am - slope * tm;
    const double r = ss_tx / (sqrt(ss_tt * ss_xx) + 1e-10);
    if (attr == 0) return slope;
    if (attr == 1) return intercept;
    if (attr == 2) return r;
    if (attr == 3) return 1.0 / (1.0 + fabs(r * sqrt(n - 2.0) / (sqrt(1.0 - r * r) + 1e-10)));
    double rss = 0.0;
    for (int i = 0; i < n; ++i) {
        const double e = a[i] - (slope * i + intercept);
        rss += e * e;
    }
    return sqrt(rss / (n - 2.0) / (ss_tt + 1e-10));
}

/* Least squares of velocity v_i = w[i+1] - w[i] on the powers p_i^m .. p_i^0 of
   position p_i = w[i] (i < n-1) by the regularised normal equations (V'V + 1e-6 I)
   c = V'v, solved with partial pivoting (torch_features_dynamical.py:87-127);
   c[0] multiplies p^m.  Returns 0, or -1 when n < 2. */
static int poly_velocity_fit(const double *w, int n, int m, double *c)
{
    if (n < 2) return -1;
    double A[7][8], pw[13];
    for (int i = 0; i <= m; ++i)
        for (int j = 0; j <= m + 1; ++j) A[i][j] = 0.0;
    double S[13], T[7];
    for (int q = 0; q <= 2 * m; ++q) S[q] = 0.0;
    for (int q = 0; q <= m; ++q) T[q] = 0.0;
    for (int i = 0; i + 1 < n; ++i) {
        const double p = w[i], v = w[i + 1] - w[i];
        pw[0] = 1.0;
        for (int q = 1; q <= 2 * m; ++q) pw[q] = pw[q - 1] * p;
        for (int q = 0; q <= 2 * m; ++q) S[q] += pw[q];
        for (int q = 0; q <= m; ++q) T[q] += pw[q] * v;
    }
    /* row a, column b of V'V: sum p^(m-a) p^(m-b) */
    for (int a = 0; a <= m; ++a) {
        for (int b = 0; b <= m; ++b) A[a][b] = S[2 * m - a - b] + (a == b ? 1e-6 : 0.0);
        A[a][m + 1] = T[m - a];
    }
    const int k = m + 1;
    for (int col = 0; col < k; ++col) {
        int piv = col;
        for (int i = col + 1; i < k; ++i)
            if (fabs(A[i][col]) > fabs(A[piv][col])) piv = i;
        if (piv != col)
            for (int j = 0; j <= k; ++j) {
                const double t = A[col][j];
                A[col][j] = A[piv][j];
                A[piv][j] = t;
            }
        for (int i = col + 1; i < k; ++i) {
            const double f = A[i][col] / A[col][col];
            for (int j = col; j <= k; ++j) A[i][j] -= f * A[col][j];
        }
    }
    for (int i = k - 1; i >= 0; --i) {
        double t = A[i][k];
        for (int j = i + 1; j < k; ++j) t -= A[i][j] * c[j];
        c[i] = t / A[i][i];
    }
    return 0;
}

/* Euclidean distance of the delay vectors starting at samples a and b */
static double lyap_dist(const double *w, long a, long b, int emb, int lag)
{
    double d2 = 0.0;
    for (int e = 0; e < emb; ++e) {
        const double df = w[a + (long)e * lag] - w[b + (long)e * lag];
        d2 += df * df;
    }
    return sqrt(d2);
}

static double window_feature(int feat, double param, double param2, const double *w, int n, double *scratch)
{
    if (n <= 0) return NAN;
    double sum = 0.0, mx = -INFINITY, mn = INFINITY;
    int any_nan = 0;
    for (int i = 0; i < n; ++i) {
        sum += w[i];
        any_nan |= isnan(w[i]);
        if (w[i] > mx) mx = w[i];
        if (w[i] < mn) mn = w[i];
    }
    if (any_nan) mx = mn = NAN; /* torch.max / torch.min propagate NaN */
    double mean = sum / n;
    double m2 = 0.0, sq = 0.0;
    for (int i = 0; i < n; ++i) {
        double d = w[i] - mean;
        m2 += d * d;
        sq += w[i] * w[i];
    }
    switch (feat) {
    case ORACLE_F_MEDIAN: { /* torch.median: the lower of the two middle values, NaN if any */
        if (any_nan) return NAN;
        memcpy(scratch, w, sizeof(double) * (size_t)n);
        qsort(scratch, (size_t)n, sizeof(double), cmp_double);
        return scratch[(n - 1) / 2];
    }
    case ORACLE_F_MEAN: return mean;
    case ORACLE_F_STD: return sqrt(m2 / n);
    case ORACLE_F_VAR: return m2 / n;
    case ORACLE_F_RMS: return sqrt(sq / n);
    case ORACLE_F_MAX: return mx;
    case ORACLE_F_ABSMAX: return fmax(fabs(mx), fabs(mn));
    case ORACLE_F_MIN: return mn;
    case ORACLE_F_DELTA: return fabs(mx - mean);
    case ORACLE_F_LOG_DELTA: return log(fabs(mx - mean) + 1e-10);
    case ORACLE_F_AMPLITUDE: return mx - mn;
    case ORACLE_F_CROSSINGS: {
        double c = 0.0;
        for (int i = 1; i < n; ++i) c += ((w[i] > param) != (w[i - 1] > param));
        return c;
    }
    case ORACLE_F_LAST: return w[n - 1];
    /* wider set: ts_torch/calculators/torch_features_statistical.py:20-27,119-163,
       torch_features_change.py:79-110, torch_features_count.py:11-33,
       torch_features_pattern.py:64-110, torch_features_autocorrelation.py:13-27 */
    case ORACLE_F_SUM: return sum;
    case ORACLE_F_ABS_ENERGY: return sq;
    case ORACLE_F_LENGTH: return (double)n;
    case ORACLE_F_VARIATION_COEFF: return sqrt(m2 / n) / (fabs(mean) + 1e-10);
    case ORACLE_F_QUANTILE: { /* torch.quantile, linear interpolation; NaN if any */
        if (any_nan) return NAN;
        memcpy(scratch, w, sizeof(double) * (size_t)n);
        qsort(scratch, (size_t)n, sizeof(double), cmp_double);
        const double pos = param * (n - 1);
        const int lo = (int)floor(pos), hi = lo + 1 < n ? lo + 1 : n - 1;
        return scratch[lo] + (scratch[hi] - scratch[lo]) * (pos - lo);
    }
    case ORACLE_F_KURTOSIS: case ORACLE_F_SKEWNESS: {
        double c2 = 0.0, c3 = 0.0, c4 = 0.0;
        for (int i = 0; i < n; ++i) {
            const double d = w[i] - mean;
            c2 += d * d;
            c3 += d * d * d;
            c4 += d * d * d * d;
        }
        c2 /= n;
        c3 /= n;
        c4 /= n;
        if (feat == ORACLE_F_KURTOSIS) {
            const double g2 = c4 / (c2 * c2 + 1e-10) - 3.0;
            return ((n - 1.0) / ((n - 2.0) * (n - 3.0) + 1e-10)) * ((n + 1.0) * g2 + 6.0);
        }
        const double g1 = c3 / (pow(c2, 1.5) + 1e-10);
        return g1 * sqrt((double)n * (n - 1.0)) / (n - 2.0 + 1e-10);
    }
    case ORACLE_F_ABS_SUM_CHANGES: case ORACLE_F_MEAN_ABS_CHANGE: {
        double a = 0.0;
        for (int i = 1; i < n; ++i) a += fabs(w[i] - w[i - 1]);
        return feat == ORACLE_F_ABS_SUM_CHANGES ? a : a / (n - 1);
    }
    case ORACLE_F_MEAN_CHANGE: return (w[n - 1] - w[0]) / (n - 1);
    case ORACLE_F_MEAN_SECOND_DERIV: return (w[n - 1] - w[n - 2] - w[1] + w[0]) / (2.0 * (n - 2));
    case ORACLE_F_COUNT_ABOVE_MEAN: case ORACLE_F_COUNT_BELOW_MEAN: {
        double c = 0.0;
        for (int i = 0; i < n; ++i) c += feat == ORACLE_F_COUNT_ABOVE_MEAN ? (w[i] > mean) : (w[i] < mean);
        return c;
    }
    case ORACLE_F_COUNT_ABOVE: case ORACLE_F_COUNT_BELOW: {
        double c = 0.0;
        for (int i = 0; i < n; ++i) c += feat == ORACLE_F_COUNT_ABOVE ? (w[i] > param) : (w[i] < param);
        return c / n;
    }
    case ORACLE_F_NUMBER_PEAKS: { /* strict local maxima with support k on each side */
        const int k = (int)param;
        double c = 0.0;
        if (2 * k >= n) return 0.0;
        for (int i = k; i < n - k; ++i) {
            int peak = 1;
            for (int j = 1; j <= k && peak; ++j) peak = (w[i] > w[i - j]) && (w[i] > w[i + j]);
            c += peak;
        }
        return c;
    }
    case ORACLE_F_AUTOCORRELATION: {
        const int lag = (int)param;
        if (lag == 0) return 1.0;
        if (lag >= n) return 0.0;
        double ac = 0.0;
        for (int i = 0; i + lag < n; ++i) ac += (w[i] - mean) * (w[i + lag] - mean);
        return ac / (m2 + 1e-10);
    }
    case ORACLE_F_RATIO_BEYOND_R_SIGMA: {
        const double sd = sqrt(m2 / n);
        double c = 0.0;
        for (int i = 0; i < n; ++i) c += fabs(w[i] - mean) > param * sd;
        return c / n;
    }
    /* torch_features_frequency.py:11-29: coefficient k of torch.fft.rfft, a direct
       DFT sum with the phase k*i/n reduced in integers */
    case ORACLE_F_SPKT_WELCH: /* torch_features_frequency.py:57-65: |X_k|^2 / n */
    case ORACLE_F_FFT_REAL: case ORACLE_F_FFT_IMAG: case ORACLE_F_FFT_ABS: case ORACLE_F_FFT_ANGLE: {
        const long k = (long)param;
        if (k > n / 2) return 0.0;
        double re = 0.0, im = 0.0;
        for (int i = 0; i < n; ++i) {
            const double ang = 6.283185307179586476925286766559 * (double)((k * i) % n) / n;
            re += w[i] * cos(ang);
            im -= w[i] * sin(ang);
        }
        if (feat == ORACLE_F_FFT_REAL) return re;
        if (feat == ORACLE_F_FFT_IMAG) return im;
        if (feat == ORACLE_F_FFT_ABS) return sqrt(re * re + im * im);
        if (feat == ORACLE_F_SPKT_WELCH) return (re * re + im * im) / n;
        return atan2(im, re);
    }
    /* torch_features_boolean.py:44-48 */
    case ORACLE_F_LARGE_STD: return sqrt(m2 / n) > param * (mx - mn) ? 1.0 : 0.0;
    /* torch_features_statistical.py:185-191 (median as torch.median: the lower middle) */
    case ORACLE_F_SYMMETRY_LOOKING: {
        if (any_nan) return NAN;
        memcpy(scratch, w, sizeof(double) * (size_t)n);
        qsort(scratch, (size_t)n, sizeof(double), cmp_double);
        return fabs(mean - scratch[(n - 1) / 2]) < param * (mx - mn) ? 1.0 : 0.0;
    }
    /* torch_features_location.py:52-65 */
    case ORACLE_F_INDEX_MASS_QUANTILE: {
        double tot = 0.0, c = 0.0;
        for (int i = 0; i < n; ++i) tot += fabs(w[i]);
        for (int i = 0; i < n; ++i) {
            c += fabs(w[i]);
            if (c >= param * tot) return (double)i / n;
        }
        return 0.0;
    }
    /* torch_features_boolean.py:23-34 */
    case ORACLE_F_HAS_DUP_MAX: case ORACLE_F_HAS_DUP_MIN: {
        if (any_nan) return 0.0;
        const double e = feat == ORACLE_F_HAS_DUP_MAX ? mx : mn;
        int c = 0;
        for (int i = 0; i < n; ++i) c += w[i] == e;
        return c > 1 ? 1.0 : 0.0;
    }
    /* torch_features_entropy_complexity.py:58-100 */
    case ORACLE_F_BINNED_ENTROPY: {
        const int bins = (int)param;
        double hb[256];
        if (mx == mn) return 0.0;
        if (bins < 1 || bins > 256) return NAN;
        for (int b = 0; b < bins; ++b) hb[b] = 0.0;
        for (int i = 0; i < n; ++i) {
            long long b = (long long)((w[i] - mn) / (mx - mn + 1e-10) * (bins - 1e-6));
            b = b < 0 ? 0 : (b > bins - 1 ? bins - 1 : b);
            hb[b] += 1.0;
        }
        double e = 0.0;
        for (int b = 0; b < bins; ++b)
            if (hb[b] > 0.0) {
                const double p = fmax(hb[b] / n, 1e-10);
                e -= p * log(p);
            }
        return e;
    }
    /* torch_features_statistical.py:166-172: mean of the k largest |x| */
    case ORACLE_F_MEAN_N_ABS_MAX: {
        const int k = (int)param < n ? (int)param : n;
        for (int i = 0; i < n; ++i) scratch[i] = fabs(w[i]);
        qsort(scratch, (size_t)n, sizeof(double), cmp_double);
        double t = 0.0;
        for (int i = 0; i < k; ++i) t += scratch[n - 1 - i];
        return t / k;
    }
    /* torch_features_advanced.py:21-81 */
    case ORACLE_F_BENFORD: {
        double f[9] = {0}, b[9], tot = 0.0, fm = 0.0, bm = 0.0;
        for (int i = 0; i < n; ++i) {
            const double v = fabs(w[i]);
            if (!(v > 0.0)) continue;
            const long long dg = (long long)floor(v / pow(10.0, floor(log10(v))));
            if (dg >= 1 && dg <= 9) {
                f[dg - 1] += 1.0;
                tot += 1.0;
            }
        }
        for (int d = 0; d < 9; ++d) {
            f[d] /= tot + 1e-10;
            fm += f[d];
            b[d] = log10(1.0 + 1.0 / (d + 1));
            bm += b[d];
        }
        fm /= 9.0;
        bm /= 9.0;
        double sfb = 0.0, sff = 0.0, sbb = 0.0;
        for (int d = 0; d < 9; ++d) {
            sfb += (f[d] - fm) * (b[d] - bm);
            sff += (f[d] - fm) * (f[d] - fm);
            sbb += (b[d] - bm) * (b[d] - bm);
        }
        const double corr = sfb / (sqrt(sff / 8.0) * sqrt(sbb / 8.0) * 9.0 + 1e-10);
        return tot >= 10.0 ? corr : 0.0;
    }
    /* torch_features_pattern.py:10-53 */
    case ORACLE_F_LONGEST_STRIKE_ABOVE: case ORACLE_F_LONGEST_STRIKE_BELOW: {
        int run = 0, best = 0;
        for (int i = 0; i < n; ++i) {
            const int on = feat == ORACLE_F_LONGEST_STRIKE_ABOVE ? w[i] > mean : w[i] < mean;
            run = on ? run + 1 : 0;
            if (run > best) best = run;
        }
        return (double)best;
    }
    /* torch_features_trend.py:11-51 (with its pseudo p-value 1 / (1 + |t|)) */
    case ORACLE_F_TREND_SLOPE: case ORACLE_F_TREND_INTERCEPT: case ORACLE_F_TREND_RVALUE:
    case ORACLE_F_TREND_PVALUE: case ORACLE_F_TREND_STDERR: {
        const double tm = 0.5 * (n - 1.0);
        double ss_tt = 0.0, ss_tx = 0.0;
        for (int i = 0; i < n; ++i) {
            ss_tt += (i - tm) * (i - tm);
            ss_tx += (i - tm) * (w[i] - mean);
        }
        const double slope = ss_tx / (ss_tt + 1e-10), intercept = mean - slope * tm;
        const double r = ss_tx / (sqrt(ss_tt * m2) + 1e-10);
        if (feat == ORACLE_F_TREND_SLOPE) return slope;
        if (feat == ORACLE_F_TREND_INTERCEPT) return intercept;
        if (feat == ORACLE_F_TREND_RVALUE) return r;
        if (feat == ORACLE_F_TREND_PVALUE) return 1.0 / (1.0 + fabs(r * sqrt(n - 2.0) / (sqrt(1.0 - r * r) + 1e-10)));
        double rss = 0.0;
        for (int i = 0; i < n; ++i) {
            const double e = w[i] - (slope * i + intercept);
            rss += e * e;
        }
        return sqrt(rss / (n - 2.0) / (ss_tt + 1e-10));
    }
    /* torch_features_location.py:11-49: index of the first (last) extreme / n */
    case ORACLE_F_FIRST_LOC_MAX: case ORACLE_F_FIRST_LOC_MIN: case ORACLE_F_LAST_LOC_MAX:
    case ORACLE_F_LAST_LOC_MIN: {
        if (any_nan) return NAN;
        const int want_max = feat == ORACLE_F_FIRST_LOC_MAX || feat == ORACLE_F_LAST_LOC_MAX;
        const int last = feat == ORACLE_F_LAST_LOC_MAX || feat == ORACLE_F_LAST_LOC_MIN;
        const double target = want_max ? mx : mn;
        int idx = -1;
        for (int i = 0; i < n; ++i)
            if (w[i] == target && (idx < 0 || last)) idx = i;
        return (double)idx / n;
    }
    /* torch_features_entropy_complexity.py:182-190 */
    case ORACLE_F_CID_CE: {
        double ce = 0.0;
        for (int i = 1; i < n; ++i) ce += (w[i] - w[i - 1]) * (w[i] - w[i - 1]);
        ce = sqrt(ce);
        return param != 0.0 ? ce / (sqrt(m2 / n) + 1e-10) : ce;
    }
    /* torch_features_advanced.py:84-90, 109-118 */
    case ORACLE_F_C3: case ORACLE_F_TIME_REVERSAL: {
        const int lag = (int)param;
        if (2 * lag >= n) return 0.0;
        const int m = n - 2 * lag;
        double a = 0.0;
        for (int i = 0; i < m; ++i) {
            const double x0 = w[i], x1 = w[i + lag], x2 = w[i + 2 * lag];
            a += feat == ORACLE_F_C3 ? x0 * x1 * x2 : x2 * x2 * x1 - x1 * x0 * x0;
        }
        return a / m;
    }
    /* torch_features_boolean.py:11-20 and torch_features_reocurrance.py:10-163: the
       window sorted ascending (NaN last, as torch.sort), then runs of equal
       neighbours; NaN equals nothing, so each NaN is a value of its own */
    case ORACLE_F_HAS_DUPLICATE: case ORACLE_F_PCT_REOCCURRING_POINTS: case ORACLE_F_PCT_REOCCURRING_VALUES:
    case ORACLE_F_SUM_REOCCURRING_POINTS: case ORACLE_F_SUM_REOCCURRING_VALUES: case ORACLE_F_RATIO_UNIQUE_VALUES: {
        memcpy(scratch, w, sizeof(double) * (size_t)n);
        qsort(scratch, (size_t)n, sizeof(double), cmp_double_nan_last);
        double dups = 0.0, in_runs = 0.0, run_starts = 0.0, sum_in_runs = 0.0, sum_run_starts = 0.0;
        for (int i = 0; i < n; ++i) {
            const int eq_prev = i > 0 && scratch[i] == scratch[i - 1];
            const int eq_next = i + 1 < n && scratch[i] == scratch[i + 1];
            dups += eq_prev;
            if (eq_prev || eq_next) {
                in_runs += 1.0;
                sum_in_runs += scratch[i];
            }
            if (eq_next && !eq_prev) {
                run_starts += 1.0;
                sum_run_starts += scratch[i];
            }
        }
        switch (feat) {
        case ORACLE_F_HAS_DUPLICATE: return dups > 0.0 ? 1.0 : 0.0;
        case ORACLE_F_PCT_REOCCURRING_POINTS: return run_starts / ((n - dups) + 1e-10);
        case ORACLE_F_PCT_REOCCURRING_VALUES: return n <= 1 ? 0.0 : in_runs / n;
        /* the reference sums sorted values times a 0/1 mask: a NaN anywhere gives NaN */
        case ORACLE_F_SUM_REOCCURRING_POINTS: return any_nan ? NAN : sum_in_runs;
        case ORACLE_F_SUM_REOCCURRING_VALUES: return any_nan ? NAN : sum_run_starts;
        default: return (n - dups) / n;
        }
    }
    /* torch_features_autocorrelation.py:31-68: lag-k autocorrelations of the centred
       window over its lag-0 sum (the reference's zero-padded FFT gives the same
       linear sums), then the Durbin-Levinson recursion with its +1e-10 guard */
    case ORACLE_F_PARTIAL_AUTOCORRELATION: {
        const int lag = (int)param;
        if (lag == 0) return 1.0;
        const int maxlag = lag < n - 1 ? lag : n - 1;
        if (maxlag < 1) return 0.0;
        double acf[ORACLE_MAX_ACF_LAG + 1], phi[ORACLE_MAX_ACF_LAG + 1], prev[ORACLE_MAX_ACF_LAG + 1];
        if (maxlag > ORACLE_MAX_ACF_LAG) return NAN;
        for (int k = 1; k <= maxlag; ++k) {
            double r = 0.0;
            for (int i = 0; i + k < n; ++i) r += (w[i] - mean) * (w[i + k] - mean);
            acf[k] = r / (m2 + 1e-10);
        }
        phi[1] = acf[1];
        for (int k = 2; k <= maxlag; ++k) {
            double num = acf[k], den = 1.0;
            for (int j = 1; j < k; ++j) {
                num -= phi[j] * acf[k - j];
                den -= phi[j] * acf[j];
            }
            const double pk = num / (den + 1e-10);
            for (int j = 1; j < k; ++j) prev[j] = phi[j];
            for (int j = 1; j < k; ++j) phi[j] = prev[j] - pk * prev[k - j];
            phi[k] = pk;
        }
        return lag <= maxlag ? phi[lag] : 0.0;
    }
    /* torch_features_autocorrelation.py:72-97: mean, lower median or population
       variance of the autocorrelations at lags 1..maxlag */
    case ORACLE_F_AGG_AUTOCORR_MEAN: case ORACLE_F_AGG_AUTOCORR_MEDIAN: case ORACLE_F_AGG_AUTOCORR_VAR: {
        const int ml = (int)param < n - 1 ? (int)param : n - 1;
        if (ml < 1 || ml > n) return NAN;
        double am = 0.0;
        for (int k = 1; k <= ml; ++k) {
            double r = 0.0;
            for (int i = 0; i + k < n; ++i) r += (w[i] - mean) * (w[i + k] - mean);
            scratch[k - 1] = r / (m2 + 1e-10);
            am += scratch[k - 1];
        }
        am /= ml;
        if (feat == ORACLE_F_AGG_AUTOCORR_MEAN) return am;
        if (feat == ORACLE_F_AGG_AUTOCORR_VAR) {
            double v = 0.0;
            for (int k = 0; k < ml; ++k) v += (scratch[k] - am) * (scratch[k] - am);
            return v / ml;
        }
        qsort(scratch, (size_t)ml, sizeof(double), cmp_double_nan_last);
        return scratch[(ml - 1) / 2];
    }
    /* torch_features_advanced.py:93-105 */
    case ORACLE_F_ENERGY_RATIO_BY_CHUNKS: {
        const int ns = (int)param, focus = (int)param2;
        const int size = ns > 0 ? n / ns : 0;
        if (size == 0) return 0.0;
        const long start = (long)focus * size;
        const long end = start + size < n ? start + size : n;
        double seg = 0.0;
        for (long i = start; i < end; ++i) seg += w[i] * w[i];
        return seg / (sq + 1e-10);
    }
    /* torch_features_count.py:37-39 */
    case ORACLE_F_COUNT_IN_RANGE: {
        double c = 0.0;
        for (int i = 0; i < n; ++i) c += (w[i] >= param && w[i] <= param2);
        return c;
    }
    /* torch_features_change.py:20-75,113-140: changes between neighbours that both
       lie in the corridor [quantile ql, quantile qh], their mean or population
       variance (0 when no change qualifies; NaN in the window gives no corridor) */
    case ORACLE_F_CHANGE_QUANTILES_MEAN: case ORACLE_F_CHANGE_QUANTILES_VAR:
    case ORACLE_F_CHANGE_QUANTILES_ABS_MEAN: case ORACLE_F_CHANGE_QUANTILES_ABS_VAR: {
        if (any_nan) return 0.0;
        memcpy(scratch, w, sizeof(double) * (size_t)n);
        qsort(scratch, (size_t)n, sizeof(double), cmp_double);
        double qv[2];
        for (int e = 0; e < 2; ++e) {
            const double pos = (e == 0 ? param : param2) * (n - 1);
            const int lo = (int)floor(pos), hi = lo + 1 < n ? lo + 1 : n - 1;
            qv[e] = scratch[lo] + (scratch[hi] - scratch[lo]) * (pos - lo);
        }
        const int isabs = feat == ORACLE_F_CHANGE_QUANTILES_ABS_MEAN || feat == ORACLE_F_CHANGE_QUANTILES_ABS_VAR;
        const int is_var = feat == ORACLE_F_CHANGE_QUANTILES_VAR || feat == ORACLE_F_CHANGE_QUANTILES_ABS_VAR;
        double s1 = 0.0, cnt = 0.0;
        for (int i = 1; i < n; ++i) {
            if (!(w[i - 1] >= qv[0] && w[i - 1] <= qv[1] && w[i] >= qv[0] && w[i] <= qv[1])) continue;
            const double d = isabs ? fabs(w[i] - w[i - 1]) : w[i] - w[i - 1];
            s1 += d;
            cnt += 1.0;
        }
        /* the reference's +1e-10 guard is added to an FP32 count (.float().sum()),
           where it vanishes: the divisor is the count itself */
        if (cnt == 0.0) return 0.0;
        const double mu = s1 / cnt;
        if (!is_var) return mu;
        double v = 0.0;
        for (int i = 1; i < n; ++i) {
            if (!(w[i - 1] >= qv[0] && w[i - 1] <= qv[1] && w[i] >= qv[0] && w[i] <= qv[1])) continue;
            const double d = isabs ? fabs(w[i] - w[i - 1]) : w[i] - w[i - 1];
            v += (d - mu) * (d - mu);
        }
        return v / cnt;
    }
    /* torch_features_autocorrelation.py:268-329 with the peak rule of
       torch_feature_utilities.py:146-218 (scipy's _local_maxima_1d): the window is
       centred and divided by its unbiased standard deviation + 1e-10, acf[k] =
       r_k / (r_0 + 1e-10) for k = 0..n-1, and a peak is the midpoint (rounded down)
       of a maximal run of equal values entered from a smaller value and left to a
       smaller one.  The first peak at index >= min_lag whose value exceeds
       peak_threshold gives the strength (its value) and the period (its index);
       none gives 0.  The lags are computed in order and the scan stops at that
       peak. */
    case ORACLE_F_ACF_PERIOD_STRENGTH: case ORACLE_F_ACF_PERIOD_LAG: {
        if (n < 2) return 0.0;
        const int min_lag = (int)param;
        const double s = sqrt(m2 / (n - 1.0)) + 1e-10, ss = s * s;
        const double r0 = m2 / ss, den = r0 + 1e-10;
        double v_run = r0 / den; /* the run holding index 0 is never a peak */
        int run_a = 0, rose = 0;
        for (int k = 1; k < n; ++k) {
            double r = 0.0;
            for (int i = 0; i + k < n; ++i) r += (w[i] - mean) * (w[i + k] - mean);
            const double v = (r / ss) / den;
            if (v == v_run) continue;
            if (rose && v < v_run) {
                const int mid = (run_a + k - 1) / 2;
                if (mid >= min_lag && v_run > param2)
                    return feat == ORACLE_F_ACF_PERIOD_STRENGTH ? v_run : (double)mid;
            }
            rose = v_run < v;
            run_a = k;
            v_run = v;
        }
        return 0.0;
    }
    /* torch_features_frequency.py:390-441: the two strongest bins of the centred
       window's power spectrum (bin 0 zeroed) at least two bins apart, the ratio of
       the second's index to the first's (ties to the lower index); 0 for a flat
       spectrum (max < 1e-10) */
    case ORACLE_F_SPECTRAL_FREQ_RATIO: {
        const int nb = n / 2 + 1;
        double *psd = (double *)malloc(sizeof(double) * (size_t)nb);
        if (!psd) return NAN;
        power_spectrum(w, n, mean, psd);
        psd[0] = 0.0;
        int first = 0;
        for (int k = 1; k < nb; ++k)
            if (psd[k] > psd[first]) first = k;
        double res = 0.0;
        if (!(psd[first] < 1e-10)) {
            int second = -1;
            for (int k = 0; k < nb; ++k)
                if (abs(k - first) >= 2 && (second < 0 || psd[k] > psd[second])) second = k;
            if (second >= 0 && first > 0) res = (double)second / first;
        }
        free(psd);
        return res;
    }
    /* torch_features_frequency.py:32-54: moments of the bin index under the
       normalised power spectrum of the (uncentred) window */
    case ORACLE_F_FFT_AGG_CENTROID: case ORACLE_F_FFT_AGG_VARIANCE: case ORACLE_F_FFT_AGG_SKEW:
    case ORACLE_F_FFT_AGG_KURTOSIS: {
        const int nb = n / 2 + 1;
        double *psd = (double *)malloc(sizeof(double) * (size_t)nb);
        if (!psd) return NAN;
        power_spectrum(w, n, 0.0, psd);
        double tot = 0.0, c = 0.0, v = 0.0, m3 = 0.0, m4 = 0.0;
        for (int k = 0; k < nb; ++k) tot += psd[k];
        for (int k = 0; k < nb; ++k) c += k * (psd[k] / (tot + 1e-10));
        for (int k = 0; k < nb; ++k) {
            const double p = psd[k] / (tot + 1e-10), d = k - c;
            v += d * d * p;
            m3 += d * d * d * p;
            m4 += d * d * d * d * p;
        }
        free(psd);
        if (feat == ORACLE_F_FFT_AGG_CENTROID) return c;
        if (feat == ORACLE_F_FFT_AGG_VARIANCE) return v;
        if (feat == ORACLE_F_FFT_AGG_SKEW) return m3 / (pow(v, 1.5) + 1e-10);
        return m4 / (v * v + 1e-10);
    }
    /* torch_features_entropy_complexity.py:97-110: entropy of the normalised power
       spectrum (uncentred window), each share clamped at 1e-10 */
    case ORACLE_F_FOURIER_ENTROPY: {
        const int nb = n / 2 + 1;
        double *psd = (double *)malloc(sizeof(double) * (size_t)nb);
        if (!psd) return NAN;
        power_spectrum(w, n, 0.0, psd);
        double tot = 0.0, h = 0.0;
        for (int k = 0; k < nb; ++k) tot += psd[k];
        for (int k = 0; k < nb; ++k) {
            double p = psd[k] / (tot + 1e-10);
            if (p < 1e-10) p = 1e-10;
            h -= p * log(p);
        }
        free(psd);
        return h;
    }
    /* torch_features_entropy_complexity.py:13-54: each embedded vector
       (w[i], w[i+tau], ..., w[i+(d-1)tau]) gets the id sum_p idx[p] * (d-1-p)!, idx
       the indices that sort it (ties in index order); the Shannon entropy of the
       ids' frequencies over log(d!).  The id is not one-to-one on permutations
       (for d = 3 only three ids occur); the reference counts these ids. */
    case ORACLE_F_PERMUTATION_ENTROPY: {
        const int tau = (int)param, d = (int)param2;
        const long np_ = (long)n - (long)(d - 1) * tau;
        if (np_ <= 0 || d < 1 || d > 7) return 0.0;
        int fact[8] = {1, 1, 2, 6, 24, 120, 720, 5040};
        double cnt[5040];
        for (int k = 0; k < fact[d]; ++k) cnt[k] = 0.0;
        for (long i = 0; i < np_; ++i) {
            int id = 0;
            for (int j = 0; j < d; ++j) {
                const double vj = w[i + (long)j * tau];
                int pos = 0;
                for (int l = 0; l < d; ++l) {
                    const double vl = w[i + (long)l * tau];
                    pos += vl < vj || (vl == vj && l < j);
                }
                id += j * fact[d - 1 - pos];
            }
            cnt[id] += 1.0;
        }
        double h = 0.0;
        for (int k = 0; k < fact[d]; ++k)
            if (cnt[k] > 0.0) {
                const double p = cnt[k] / np_;
                h -= p * log(p);
            }
        return fact[d] > 1 ? h / log((double)fact[d]) : h;
    }
    /* torch_features_entropy_complexity.py:141-178: the window cut into `bins`
       equal bins over [min, max + 1e-10), then parsed into phrases, each the
       shortest substring from the current position not seen as a phrase before
       (so every phrase extends an earlier one by one symbol: an LZ78 trie); the
       phrase count over n / log n.  A final substring already seen adds nothing. */
    case ORACLE_F_LEMPEL_ZIV: {
        const int bins = (int)param;
        const double range = (mx - mn) + 1e-10;
        int *sym = (int *)malloc(sizeof(int) * (size_t)n);
        int *child = (int *)malloc(sizeof(int) * (size_t)(n + 1) * (size_t)bins);
        if (!sym || !child) {
            free(sym);
            free(child);
            return NAN;
        }
        for (int i = 0; i < n; ++i) {
            long b = (long)((w[i] - mn) / range * bins);
            sym[i] = (int)(b < 0 ? 0 : (b > bins - 1 ? bins - 1 : b));
        }
        for (long q = 0; q < (long)(n + 1) * bins; ++q) child[q] = -1;
        int nodes = 1, complexity = 0;
        long i = 0;
        while (i < n) {
            int node = 0;
            long len = 1;
            while (i + len <= n) {
                const int c = sym[i + len - 1];
                const int nx = child[(long)node * bins + c];
                if (nx < 0) {
                    child[(long)node * bins + c] = nodes++;
                    ++complexity;
                    break;
                }
                node = nx;
                ++len;
            }
            i += len;
        }
        free(sym);
        free(child);
        const double b_n = n > 1 ? n / (log((double)n) + 1e-10) : 1.0;
        return complexity / b_n;
    }
    /* torch_features_trend.py:60-83: linear trend of the chunk aggregates (mean,
       population variance, min or max of consecutive chunks of chunk_size samples;
       a partial last chunk is dropped); 0 with fewer than two chunks */
    case ORACLE_F_AGG_TREND_MEAN: case ORACLE_F_AGG_TREND_VAR: case ORACLE_F_AGG_TREND_MIN:
    case ORACLE_F_AGG_TREND_MAX: {
        const int cs = (int)param, nc = cs > 0 ? n / cs : 0;
        if (nc < 2) return 0.0;
        for (int c = 0; c < nc; ++c) {
            const double *q = w + (long)c * cs;
            double s1 = 0.0, lo = q[0], hi = q[0];
            for (int i = 0; i < cs; ++i) {
                s1 += q[i];
                if (q[i] < lo) lo = q[i];
                if (q[i] > hi) hi = q[i];
            }
            const double cm = s1 / cs;
            double v = 0.0;
            for (int i = 0; i < cs; ++i) v += (q[i] - cm) * (q[i] - cm);
            scratch[c] = feat == ORACLE_F_AGG_TREND_MEAN ? cm
                         : feat == ORACLE_F_AGG_TREND_VAR ? v / cs
                         : feat == ORACLE_F_AGG_TREND_MIN ? lo : hi;
        }
        return trend_attr(scratch, nc, (int)param2);
    }
    /* torch_features_trend.py:86-131: Yule-Walker, R phi = r with R_ij =
       acf[|i-j|] + 1e-6 delta_ij and r = acf[1..k], acf[k] = sum d_i d_(i+k) /
       (sum d_i^2 + 1e-10); coefficient `coeff` of phi (0 when coeff >= k), solved by
       Gaussian elimination with partial pivoting */
    case ORACLE_F_AR_COEFFICIENT: {
        const int k = (int)param, coeff = (int)param2;
        if (coeff >= k || k < 1 || k > 10) return 0.0;
        double acf[11], R[10][11];
        for (int l = 0; l <= k; ++l) {
            double r = 0.0;
            for (int i = 0; i + l < n; ++i) r += (w[i] - mean) * (w[i + l] - mean);
            acf[l] = r / (m2 + 1e-10);
        }
        for (int i = 0; i < k; ++i) {
            for (int j = 0; j < k; ++j) R[i][j] = acf[abs(i - j)] + (i == j ? 1e-6 : 0.0);
            R[i][k] = acf[i + 1];
        }
        for (int c = 0; c < k; ++c) {
            int piv = c;
            for (int i = c + 1; i < k; ++i)
                if (fabs(R[i][c]) > fabs(R[piv][c])) piv = i;
            if (piv != c)
                for (int j = 0; j <= k; ++j) {
                    const double t = R[c][j];
                    R[c][j] = R[piv][j];
                    R[piv][j] = t;
                }
            for (int i = c + 1; i < k; ++i) {
                const double f = R[i][c] / R[c][c];
                for (int j = c; j <= k; ++j) R[i][j] -= f * R[c][j];
            }
        }
        double phi[10];
        for (int i = k - 1; i >= 0; --i) {
            double t = R[i][k];
            for (int j = i + 1; j < k; ++j) t -= R[i][j] * phi[j];
            phi[i] = t / R[i][i];
        }
        return phi[coeff];
    }
    /* torch_features_frequency.py:71-127: the Ricker wavelet of width w on t = -4w..4w,
       (2 / (sqrt(3w) pi^0.25)) (1 - (t/w)^2) exp(-t^2 / (2 w^2)) -- the reference forms
       the prefactor in FP32 (its sqrt of a default-dtype tensor), so it is rounded
       the same way here -- correlated with the window padded by 4w samples
       (reflected without repeating the edge, or replicated when n < 4w); the output
       at index coeff (0 past the end or when w is not one of the widths) */
    case ORACLE_F_CWT: {
        const int wd = (int)param, coeff = (int)param2;
        if (coeff < 0 || coeff >= n || wd < 1) return 0.0;
        const float s32 = sqrtf((float)(3.0 * wd));
        const double pi = 3.14159265358979323846;
        const float pref32 = 2.0f / (s32 * (float)pow(pi, 0.25));
        const double pref = (double)pref32, sig = (double)wd;
        const int pad = 4 * wd;
        double acc = 0.0;
        for (int j = 0; j <= 8 * wd; ++j) {
            const double t = (double)(j - pad);
            const double psi = pref * (1.0 - (t / sig) * (t / sig)) * exp(-(t * t) / (2.0 * sig * sig));
            long q = (long)coeff + j - pad;
            if (n >= pad) {
                if (q < 0) q = -q;
                if (q >= n) q = 2L * (n - 1) - q;
            } else {
                q = q < 0 ? 0 : (q >= n ? n - 1 : q);
            }
            acc += w[q] * psi;
        }
        return acc;
    }
    /* torch_features_dynamical.py:87-127 (r unused, as in the reference) */
    case ORACLE_F_FRIEDRICH: {
        const int m = (int)param, coeff = (int)param2;
        double c[7];
        if (m < 0 || m > 6 || poly_velocity_fit(w, n, m, c) != 0) return 0.0;
        return coeff <= m ? c[coeff] : 0.0;
    }
    /* torch_features_dynamical.py:131-174: the fitted velocity at each position in
       time order; the largest position p_i (i < n-2) where the fit changes sign
       strictly between i and i+1, 0 if none */
    case ORACLE_F_LANGEVIN: {
        const int m = (int)param;
        double c[7];
        if (m < 0 || m > 6 || poly_velocity_fit(w, n, m, c) != 0) return 0.0;
        double best = -INFINITY, prev = 0.0;
        for (int i = 0; i + 1 < n; ++i) {
            double f = 0.0;
            for (int q = 0; q <= m; ++q) f = f * w[i] + c[q];
            if (i > 0 && prev * f < 0.0 && w[i - 1] > best) best = w[i - 1];
            prev = f;
        }
        return best == -INFINITY ? 0.0 : best;
    }
    /* torch_features_trend.py:134-169: least squares of the first difference
       d_i = w[i+1] - w[i] on the lagged value w[i] (i < n-1), t = beta / (se + 1e-10)
       with se = sqrt(rss / (n - 3)) / (sqrt(ss_xx) + 1e-10); pvalue = 1 / (1 + |t|);
       usedlag is 1 */
    case ORACLE_F_ADF_TESTSTAT: case ORACLE_F_ADF_PVALUE: case ORACLE_F_ADF_USEDLAG: {
        if (feat == ORACLE_F_ADF_USEDLAG) return 1.0;
        const int nm = n - 1;
        double xm = 0.0, ym = 0.0;
        for (int i = 0; i < nm; ++i) {
            xm += w[i];
            ym += w[i + 1] - w[i];
        }
        xm /= nm;
        ym /= nm;
        double sxx = 0.0, sxy = 0.0;
        for (int i = 0; i < nm; ++i) {
            sxx += (w[i] - xm) * (w[i] - xm);
            sxy += (w[i] - xm) * ((w[i + 1] - w[i]) - ym);
        }
        const double beta = sxy / (sxx + 1e-10);
        double rss = 0.0;
        for (int i = 0; i < nm; ++i) {
            const double e = (w[i + 1] - w[i]) - (ym + beta * (w[i] - xm));
            rss += e * e;
        }
        const double se = sqrt(rss / (n - 3.0)) / (sqrt(sxx) + 1e-10);
        const double t = beta / (se + 1e-10);
        return feat == ORACLE_F_ADF_TESTSTAT ? t : 1.0 / (1.0 + fabs(t));
    }
    /* torch_features_pattern.py:154-188: for each width 1..max_width with 2 width < n,
       the samples i in [width, n - width) equal to the maximum of w[i-width..i+width]
       (a NaN in that neighbourhood rules the sample out: max pooling propagates
       NaN); the count averaged over those widths (0 if none) */
    case ORACLE_F_NUMBER_CWT_PEAKS: {
        const int mw = (int)param;
        double tot = 0.0;
        int nw = 0;
        for (int wd = 1; wd <= mw; ++wd) {
            if (!(2 * wd < n)) continue;
            ++nw;
            for (int i = wd; i < n - wd; ++i) {
                double mxl = w[i - wd];
                int nan_in = isnan(mxl) != 0;
                for (int j = i - wd + 1; j <= i + wd; ++j) {
                    nan_in |= isnan(w[j]) != 0;
                    if (w[j] > mxl) mxl = w[j];
                }
                tot += !nan_in && w[i] == mxl;
            }
        }
        return nw > 0 ? tot / nw : 0.0;
    }
    /* ts_torch/torch_corr_dim.py:17-110 (Grassberger-Procaccia, as the reference
       states it): delay vectors of emb_dim samples `lag` apart; n_rvals radii
       exp(log(0.1 sd + 1e-10) + a_k (log(0.5 sd + 1e-10) - log(0.1 sd + 1e-10))), sd
       the unbiased standard deviation, formed in FP32 as the reference's type
       promotion does (a_k = torch.linspace(0, 1, n_rvals) in FP32: fma(step, k, 0)
       for the first half, fma(-step, n_rvals - 1 - k, 1) for the rest); C(r_k) = the
       share of ordered pairs of distinct vectors within r_k (Euclidean); the least-
       squares slope of log C on log r over the radii with C > 0, NaN with fewer than
       two or a degenerate fit */
    case ORACLE_F_CORR_DIM: {
        const int emb = (int)param, packed = (int)param2;
        const int lag = packed / 1024, nr = packed % 1024;
        const long M = (long)n - (long)(emb - 1) * lag;
        if (M < 2 || nr < 1 || emb < 1 || lag < 1) return NAN;
        const double sd = sqrt(m2 / (n - 1.0));
        const double lmin = log(0.1 * sd + 1e-10), lmax = log(0.5 * sd + 1e-10);
        const float ld = (float)(lmax - lmin), lmin32 = (float)lmin;
        const float step = nr > 1 ? 1.0f / (float)(nr - 1) : 0.0f;
        double *rv = (double *)malloc(sizeof(double) * (size_t)nr);
        double *cnt = (double *)calloc((size_t)nr, sizeof(double));
        if (!rv || !cnt) {
            free(rv);
            free(cnt);
            return NAN;
        }
        for (int k = 0; k < nr; ++k) {
            const float a = k < nr / 2 ? fmaf(step, (float)k, 0.0f) : fmaf(-step, (float)(nr - 1 - k), 1.0f);
            const float prod = a * ld;
            const float arg = lmin32 + prod;
            rv[k] = (double)(float)exp((double)arg);
        }
        for (long i = 0; i < M; ++i)
            for (long j = i + 1; j < M; ++j) {
                double d2 = 0.0;
                for (int e = 0; e < emb; ++e) {
                    const double df = w[i + (long)e * lag] - w[j + (long)e * lag];
                    d2 += df * df;
                }
                const double dist = sqrt(d2);
                if (!(dist <= rv[nr - 1])) continue;
                int lo = 0, hi = nr - 1; /* smallest k with dist <= rv[k] */
                while (lo < hi) {
                    const int mid = (lo + hi) / 2;
                    if (dist <= rv[mid]) hi = mid;
                    else lo = mid + 1;
                }
                cnt[lo] += 2.0;
            }
        /* the fit in centred form (n sum (r - mr)^2 equals the reference's
           n sum r^2 - (sum r)^2, but is exactly 0 when all radii coincide) */
        double acc = 0.0, nv = 0.0, sr = 0.0, sc = 0.0;
        for (int k = 0; k < nr; ++k) {
            acc += cnt[k];
            cnt[k] = acc / ((double)M * (double)(M - 1)); /* C(r_k) */
            if (!(cnt[k] > 0.0)) continue;
            nv += 1.0;
            sr += log(rv[k]);
            sc += log(cnt[k] + 1e-30);
        }
        double srr = 0.0, src = 0.0;
        for (int k = 0; k < nr; ++k) {
            if (!(cnt[k] > 0.0)) continue;
            const double dr = log(rv[k]) - sr / nv, dc = log(cnt[k] + 1e-30) - sc / nv;
            srr += dr * dr;
            src += dr * dc;
        }
        free(rv);
        free(cnt);
        const double den = nv * srr;
        return (nv >= 2.0 && fabs(den) > 1e-10) ? (nv * src) / den : NAN;
    }
    /* ts_torch/torch_lyapunov_r.py (Rosenstein, as the reference states it):
       min_tsep = ceil(1 / mean frequency) of the power spectrum of the window
       zero-padded to 2n-1 (bins k >= 1, frequency k / (2n-1)), clamped to
       [1, floor(n / 4)]; delay vectors of emb_dim samples `lag` apart; each of the
       first ntraj = max(M - L + 1, 1) vectors takes as neighbour the first nearest
       one among them more than min_tsep away (index 0 if none); div[k] = mean over
       i of log d(i + k, nb(i) + k) over pairs inside the orbit with d > 0 (a pair
       within min_tsep counts as +inf), stored in FP32 as the reference's buffer
       is; the least-squares slope of div on k = 0..L-1 over its finite entries */
    case ORACLE_F_LYAP_R: {
        const int emb = (int)param / 1024, L = (int)param % 1024, lag = (int)param2;
        const long M = (long)n - (long)(emb - 1) * lag;
        if (M < 1 || emb < 1 || L < 1 || lag < 1) return NAN;
        const long N2 = 2L * n - 1;
        const double two_pi = 6.283185307179586476925286766559;
        double sfp = 0.0, sp = 0.0;
        for (long k = 1; k <= N2 / 2; ++k) {
            double re = 0.0, im = 0.0;
            long ph = 0;
            for (int i = 0; i < n; ++i) {
                const double ang = two_pi * (double)ph / N2;
                re += w[i] * cos(ang);
                im -= w[i] * sin(ang);
                ph += k;
                if (ph >= N2) ph -= N2;
            }
            const double p = re * re + im * im;
            sfp += ((double)k / N2) * p;
            sp += p;
        }
        const double mf = sfp / (sp + 1e-10);
        long tsep = (long)ceil(1.0 / (mf + 1e-10));
        const long maxt = (long)(0.25 * n);
        if (tsep > maxt) tsep = maxt;
        if (tsep < 1) tsep = 1;
        const long ntraj = M - L + 1 > 1 ? M - L + 1 : 1;
#define LYAP_DIST(a, b) (labs((a) - (b)) <= tsep ? INFINITY : lyap_dist(w, (a), (b), emb, lag))
        long *nb = (long *)malloc(sizeof(long) * (size_t)ntraj);
        if (!nb) return NAN;
        for (long i = 0; i < ntraj; ++i) {
            double best = INFINITY;
            long bj = 0;
            for (long j = 0; j < ntraj; ++j) {
                const double d = LYAP_DIST(i, j);
                if (d < best) {
                    best = d;
                    bj = j;
                }
            }
            nb[i] = bj;
        }
        double nf = 0.0, sk = 0.0, sd = 0.0, skk = 0.0, skd = 0.0;
        for (int k = 0; k < L; ++k) {
            double acc = 0.0, cnt = 0.0;
            for (long i = 0; i < ntraj; ++i) {
                if (i + k >= M || nb[i] + k >= M) continue;
                const double d = LYAP_DIST(i + k, nb[i] + k);
                if (!(d > 0.0)) continue;
                acc += log(d);
                cnt += 1.0;
            }
            const double div = (double)(float)(cnt > 0.0 ? acc / cnt : NAN);
            if (!isfinite(div)) continue;
            nf += 1.0;
            sk += k;
            sd += div;
            skk += (double)k * k;
            skd += k * div;
        }
#undef LYAP_DIST
        free(nb);
        const double den = nf * skk - sk * sk;
        return (nf >= 2.0 && fabs(den) > 1e-10) ? (nf * skd - sk * sd) / den : NAN;
    }
    /* torch_features_boolean.py:37-41 */
    case ORACLE_F_VAR_LARGER_THAN_STD: return sqrt(m2 / n) > 1.0 ? 1.0 : 0.0;
    /* torch_features_count.py:42-45 */
    case ORACLE_F_COUNT_VALUE: {
        double c = 0.0;
        for (int i = 0; i < n; ++i) c += w[i] == param;
        return c;
    }
    default: return NAN;
    }
}

/* ---- initial step (Hairer, Norsett & Wanner II.4) ------------------------ */
static double initial_step(int sys, const double *p, const double *y0, const double *f0, int dim,
                           double t0, double rtol, double atol, const oracle_aux *aux,
                           double *ytmp, double *ftmp)
{
    double d0 = 0.0, d1 = 0.0;
    for (int i = 0; i < dim; ++i) {
        double sc = atol + fabs(y0[i]) * rtol;
        double r0 = y0[i] / sc, r1 = f0[i] / sc;
        d0 += r0 * r0;
        d1 += r1 * r1;
    }
    d0 = sqrt(d0 / dim);
    d1 = sqrt(d1 / dim);
    double h0 = (d0 < 1e-5 || d1 < 1e-5) ? 1e-6 : 0.01 * d0 / d1;
    for (int i = 0; i < dim; ++i) ytmp[i] = y0[i] + h0 * f0[i];
    rhs(sys, t0 + h0, ytmp, ftmp, p, dim, aux);
    double d2 = 0.0;
    for (int i = 0; i < dim; ++i) {
        double sc = atol + fabs(y0[i]) * rtol;
        double r = (ftmp[i] - f0[i]) / sc;
        d2 += r * r;
    }
    d2 = sqrt(d2 / dim) / h0;
    double h1 = (d1 <= 1e-15 && d2 <= 1e-15) ? fmax(1e-6, h0 * 1e-3) : pow(0.01 / fmax(d1, d2), 0.2);
    return fmin(100.0 * h0, h1);
}

/* ---- one trajectory ------------------------------------------------------ */
typedef struct {
    double *y, *ynew, *ystage, *k[7], *ia, *ib, *ic, *win, *scratch, *ytmp, *ftmp;
} work_t;

static int solve_one(const oracle_problem *pb, const double *y0, const double *p, work_t *w,
                     double *feat_out, double *y_final, double *y_full, int64_t traj,
                     int64_t n_traj, int64_t *steps_out, int64_t *accepted_out)
{
    const int dim = pb->dim;
    const int ns = pb->n_save;
    const int wb = pb->win_begin;
    const int nwin = ns - wb;
    double *y = w->y, *yn = w->ynew, *ys = w->ystage;
    int k1 = 0, k7 = 6;
    int status = ORACLE_OK;
    memcpy(y, y0, sizeof(double) * (size_t)dim);
    double t = pb->t0;
    int si = 0;
    rhs(pb->system, t, y, w->k[k1], p, dim, pb->aux);
    double dt = initial_step(pb->system, p, y0, w->k[k1], dim, t, pb->rtol, pb->atol, pb->aux,
                             w->ytmp, w->ftmp);
    int64_t steps = 0, accepted = 0;
#define STORE_SAVE(idx, src)                                                                     \
    do {                                                                                         \
        if ((idx) >= wb) memcpy(w->win + (size_t)((idx) - wb) * dim, (src), sizeof(double) * dim); \
        if (y_full)                                                                              \
            memcpy(y_full + ((size_t)(idx) * (size_t)n_traj + (size_t)traj) * dim, (src),        \
                   sizeof(double) * dim);                                                        \
    } while (0)

    while (t < pb->t1 && steps < pb->max_steps) {
        steps++;
        if (t + dt > pb->t1) dt = pb->t1 - t;
        if (dt <= 0.0) break;
        if (t + dt == t) { status = ORACLE_DT_UNDERFLOW; break; }
        double *K1 = w->k[k1], *K2 = w->k[1], *K3 = w->k[2], *K4 = w->k[3], *K5 = w->k[4],
               *K6 = w->k[5], *K7 = w->k[k7];
        for (int i = 0; i < dim; ++i) ys[i] = y[i] + dt * A21 * K1[i];
        rhs(pb->system, t + C2 * dt, ys, K2, p, dim, pb->aux);
        for (int i = 0; i < dim; ++i) ys[i] = y[i] + dt * (A31 * K1[i] + A32 * K2[i]);
        rhs(pb->system, t + C3 * dt, ys, K3, p, dim, pb->aux);
        for (int i = 0; i < dim; ++i) ys[i] = y[i] + dt * (A41 * K1[i] + A42 * K2[i] + A43 * K3[i]);
        rhs(pb->system, t + C4 * dt, ys, K4, p, dim, pb->aux);
        for (int i = 0; i < dim; ++i)
            ys[i] = y[i] + dt * (A51 * K1[i] + A52 * K2[i] + A53 * K3[i] + A54 * K4[i]);
        rhs(pb->system, t + C5 * dt, ys, K5, p, dim, pb->aux);
        for (int i = 0; i < dim; ++i)
            ys[i] = y[i] + dt * (A61 * K1[i] + A62 * K2[i] + A63 * K3[i] + A64 * K4[i] + A65 * K5[i]);
        rhs(pb->system, t + dt, ys, K6, p, dim, pb->aux);
        for (int i = 0; i < dim; ++i)
            yn[i] = y[i] + dt * (B1 * K1[i] + B3 * K3[i] + B4 * K4[i] + B5 * K5[i] + B6 * K6[i]);
        rhs(pb->system, t + dt, yn, K7, p, dim, pb->aux);

        double err = 0.0;
        for (int i = 0; i < dim; ++i) {
            double e = dt * (E1 * K1[i] + E3 * K3[i] + E4 * K4[i] + E5 * K5[i] + E6 * K6[i] + E7 * K7[i]);
            double sc = pb->atol + pb->rtol * fmax(fabs(y[i]), fabs(yn[i]));
            double r = e / sc;
            err += r * r;
        }
        err = sqrt(err / dim);
        if (!isfinite(err)) { status = ORACLE_NONFINITE; break; }

        if (err <= 1.0) {
            double tn = t + dt;
            accepted++;
            if (si < ns && pb->save_ts[si] <= tn + 1e-12) {
                for (int i = 0; i < dim; ++i) {
                    double ym = y[i] + dt * (M1 * K1[i] + M3 * K3[i] + M4 * K4[i] + M5 * K5[i] +
                                             M6 * K6[i] + M7 * K7[i]);
                    w->ia[i] = 2.0 * dt * (K7[i] - K1[i]) - 8.0 * (yn[i] + y[i]) + 16.0 * ym;
                    w->ib[i] = dt * (5.0 * K1[i] - 3.0 * K7[i]) + 18.0 * y[i] + 14.0 * yn[i] - 32.0 * ym;
                    w->ic[i] = dt * (K7[i] - 4.0 * K1[i]) - 11.0 * y[i] - 5.0 * yn[i] + 16.0 * ym;
                }
                while (si < ns && pb->save_ts[si] <= tn + 1e-12) {
                    if (pb->save_ts[si] <= t + 1e-12) {
                        STORE_SAVE(si, y);
                    } else {
                        double x = (pb->save_ts[si] - t) / dt;
                        for (int i = 0; i < dim; ++i)
                            w->ytmp[i] = y[i] + x * (dt * K1[i] + x * (w->ic[i] + x * (w->ib[i] + x * w->ia[i])));
                        STORE_SAVE(si, w->ytmp);
                    }
                    si++;
                }
            }
            memcpy(y, yn, sizeof(double) * (size_t)dim);
            t = tn;
            int tmp = k1; k1 = k7; k7 = tmp;
            if (pb->unbounded_thr > 0.0) {
                double m = 0.0;
                for (int i = 0; i < dim; ++i) m = fmax(m, fabs(y[i]));
                if (m >= pb->unbounded_thr) { status = ORACLE_UNBOUNDED; break; }
            }
        }
        double dfac = (err <= 1.0) ? 1.0 : MIN_FACTOR;
        double fac = (err == 0.0) ? MAX_FACTOR : fmin(MAX_FACTOR, fmax(dfac, SAFETY * pow(err, -0.2)));
        dt *= fac;
    }
    if (status == ORACLE_OK && t < pb->t1 && steps >= pb->max_steps) status = ORACLE_MAX_STEPS;

    /* remaining save points: last state (Zig semantics), +inf after a stop event */
    for (; si < ns; ++si) {
        if (status == ORACLE_UNBOUNDED) {
            for (int i = 0; i < dim; ++i) w->ytmp[i] = INFINITY;
            STORE_SAVE(si, w->ytmp);
        } else {
            STORE_SAVE(si, y);
        }
    }
#undef STORE_SAVE
    if (y_final) memcpy(y_final, y, sizeof(double) * (size_t)dim);
    if (steps_out) *steps_out = steps;
    if (accepted_out) *accepted_out = accepted;

    for (int f = 0; feat_out && f < pb->n_features; ++f) {
        int state = pb->feat_state[f];
        for (int j = 0; j < nwin; ++j) w->scratch[nwin + j] = w->win[(size_t)j * dim + state];
        feat_out[f] = window_feature(pb->feat_kind[f], pb->feat_param ? pb->feat_param[f] : 0.0,
                                     pb->feat_param2 ? pb->feat_param2[f] : 0.0, w->scratch + nwin, nwin,
                                     w->scratch);
    }
    return status;
}

int oracle_solve_batch(const oracle_problem *pb, const double *y0s, int64_t n_traj,
                       const double *params, const int32_t *param_index, double *features_out,
                       int32_t *status_out, double *y_final, double *y_full, int64_t *steps_out,
                       int64_t *accepted_out, int n_threads)
{
    if (!pb || pb->dim <= 0 || n_traj < 0 || pb->n_save < 0 || pb->win_begin < 0 ||
        pb->win_begin > pb->n_save)
        return ORACLE_EINVAL;
    const int dim = pb->dim;
    const int nwin = pb->n_save - pb->win_begin;
    int err_flag = 0;
#ifdef _OPENMP
    if (n_threads <= 0) n_threads = omp_get_max_threads();
#pragma omp parallel num_threads(n_threads)
#endif
    {
        work_t w;
        size_t per = (size_t)dim;
        double *buf = (double *)calloc(per * 18 + (size_t)nwin * dim + 2 * (size_t)nwin + 8, sizeof(double));
        if (!buf) {
#ifdef _OPENMP
#pragma omp atomic write
#endif
            err_flag = 1;
        } else {
            double *q = buf;
            w.y = q; q += per; w.ynew = q; q += per; w.ystage = q; q += per;
            for (int s = 0; s < 7; ++s) { w.k[s] = q; q += per; }
            w.ia = q; q += per; w.ib = q; q += per; w.ic = q; q += per;
            w.ytmp = q; q += per; w.ftmp = q; q += per;
            w.win = q; q += (size_t)nwin * dim;
            w.scratch = q;
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 16)
#endif
            for (int64_t j = 0; j < n_traj; ++j) {
                int64_t prow = param_index ? param_index[j] : 0;
                int st = solve_one(pb, y0s + (size_t)j * dim, params + (size_t)prow * pb->n_params, &w,
                                   features_out ? features_out + (size_t)j * pb->n_features : NULL,
                                   y_final ? y_final + (size_t)j * dim : NULL, y_full, j, n_traj,
                                   steps_out ? steps_out + j : NULL, accepted_out ? accepted_out + j : NULL);
                if (status_out) status_out[j] = st;
            }
            free(buf);
        }
    }
    return err_flag ? ORACLE_ENOMEM : ORACLE_OK;
}

/* Feature of one stored window (used to pin the statistics against the reference's calculators). */
double oracle_window_feature(int kind, double param, const double *w, int n)
{
    return oracle_window_feature2(kind, param, 0.0, w, n);
}

double oracle_window_feature2(int kind, double param, double param2, const double *w, int n)
{
    double *scratch = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    if (!scratch) return NAN;
    double v = window_feature(kind, param, param2, w, n, scratch);
    free(scratch);
    return v;
}
