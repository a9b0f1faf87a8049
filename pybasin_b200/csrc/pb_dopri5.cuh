// Per-lane adaptive Dormand-Prince 5(4) integrator with dense output fused
// into streaming window statistics.
//
// One CUDA thread owns one trajectory at a time; its state, stages and
// statistics live in registers.  The algorithm (tableau, Shampine error
// estimate, torchdiffeq-style control and 4th-order dense output) is the one
// of the reference's native solver, src/zigode/src/solver/dopri5_generic.zig:
//   step and stages      :130-183
//   RMS error norm       :185-192
//   dense output         :194-221
//   FSAL swap            :223-225
//   step-size control    :228-235 (safety 0.9, min 0.2, max 10, no shrink on accept)
//   initial step size    :270-321 (Hairer, Norsett & Wanner II.4)
//   tail fill            :238-241
// Statistics follow src/pybasin/ts_torch/calculators/torch_features_statistical.py
// (:30-110, :307-318) and torch_features_pattern.py:56-60, evaluated as
// streaming (shifted-sum) reductions over the save points of the window
// instead of over a stored (T, B, S) tensor.
#pragma once
#include <cuda_runtime.h>
#include <math_constants.h>
#include <stdint.h>

#include "pb_rhs.cuh"
#include "pybasin_b200.h"

namespace pb {

// ---- Dormand-Prince tableau (published method constants) -----------------
namespace dp {
constexpr double a21 = 1.0 / 5.0;
constexpr double a31 = 3.0 / 40.0, a32 = 9.0 / 40.0;
constexpr double a41 = 44.0 / 45.0, a42 = -56.0 / 15.0, a43 = 32.0 / 9.0;
constexpr double a51 = 19372.0 / 6561.0, a52 = -25360.0 / 2187.0, a53 = 64448.0 / 6561.0,
                 a54 = -212.0 / 729.0;
constexpr double a61 = 9017.0 / 3168.0, a62 = -355.0 / 33.0, a63 = 46732.0 / 5247.0,
                 a64 = 49.0 / 176.0, a65 = -5103.0 / 18656.0;
constexpr double b1 = 35.0 / 384.0, b3 = 500.0 / 1113.0, b4 = 125.0 / 192.0,
                 b5 = -2187.0 / 6784.0, b6 = 11.0 / 84.0;
constexpr double c2 = 1.0 / 5.0, c3 = 3.0 / 10.0, c4 = 4.0 / 5.0, c5 = 8.0 / 9.0;
constexpr double e1 = 35.0 / 384.0 - 1951.0 / 21600.0;
constexpr double e3 = 500.0 / 1113.0 - 22642.0 / 50085.0;
constexpr double e4 = 125.0 / 192.0 - 451.0 / 720.0;
constexpr double e5 = -2187.0 / 6784.0 - -12231.0 / 42400.0;
constexpr double e6 = 11.0 / 84.0 - 649.0 / 6300.0;
constexpr double e7 = -1.0 / 60.0;
constexpr double m1 = 6025192743.0 / 30085553152.0 / 2.0;
constexpr double m3 = 51252292925.0 / 65400821598.0 / 2.0;
constexpr double m4 = -2691868925.0 / 45128329728.0 / 2.0;
constexpr double m5 = 187940372067.0 / 1594534317056.0 / 2.0;
constexpr double m6 = -1776094331.0 / 19743644256.0 / 2.0;
constexpr double m7 = 11237099.0 / 235043384.0 / 2.0;
constexpr double safety = 0.9, min_factor = 0.2, max_factor = 10.0;
constexpr double save_slack = 1e-12;  // dopri5_generic.zig:197,205,207
}  // namespace dp

// Select arr[idx] for a runtime idx without dynamic register indexing.
template <int N, class T>
__device__ __forceinline__ T pick(const T (&arr)[N], int idx)
{
    T v = arr[0];
#pragma unroll
    for (int i = 1; i < N; ++i) v = (idx == i) ? arr[i] : v;
    return v;
}

template <class Sys, class R>
struct Lane {
    static constexpr int S = Sys::S;
    R y[S];
    R yc[S];  // Kahan compensation of y (mixed precision only)
    R k1[S];
    R p[Sys::NP];
    double t, dt;
    int64_t steps;
    int si;            // next save index
    double next_save;  // save_ts[si] (or +inf past the end)
    int status;
    // window statistics
    int nsamp;
    unsigned nan_mask;
    double shift[S], s1[S], s2[S];
    R mn[S], mx[S], last[S];
    int cross_cnt[PB_MAX_CROSSING];
    unsigned cross_prev;  // bit j: previous sample of crossing slot j was above its level
};

__device__ __forceinline__ double load_save(const pb_solve_args& a, int si)
{
    return si < a.n_save ? __ldg(a.save_ts + si) : CUDART_INF;
}

template <class Sys, class R, bool MIXED>
struct Integrator {
    static constexpr int S = Sys::S;
    using L_t = Lane<Sys, R>;

    // ---- one save point: window statistics, optional full output, median window
    __device__ static void record(L_t& L, const R (&v)[S], int64_t traj, const pb_solve_args& a)
    {
        if (L.si >= a.win_begin) {
            const int n = L.nsamp;
#pragma unroll
            for (int s = 0; s < S; ++s) {
                const double x = static_cast<double>(v[s]);
                if (n == 0) {
                    L.shift[s] = isfinite(x) ? x : 0.0;
                    L.mn[s] = v[s];
                    L.mx[s] = v[s];
                }
                const double d = x - L.shift[s];
                L.s1[s] += d;
                L.s2[s] += d * d;
                L.mn[s] = fmin(L.mn[s], v[s]);
                L.mx[s] = fmax(L.mx[s], v[s]);
                if (isnan(x)) L.nan_mask |= 1u << s;
                L.last[s] = v[s];
            }
            int j = 0, med = 0;
            for (int c = 0; c < a.n_features; ++c) {
                const int kind = a.feat_kind[c];
                if (kind == PB_FEAT_CROSSINGS && j < PB_MAX_CROSSING) {
                    const bool above = static_cast<double>(pick(v, a.feat_state[c])) > a.feat_param[c];
                    const bool prev = (L.cross_prev >> j) & 1u;
                    if (n > 0 && above != prev) {
#pragma unroll
                        for (int q = 0; q < PB_MAX_CROSSING; ++q) L.cross_cnt[q] += (q == j);
                    }
                    L.cross_prev = (L.cross_prev & ~(1u << j)) | (static_cast<unsigned>(above) << j);
                    ++j;
                } else if (kind == PB_FEAT_MEDIAN) {
                    const int64_t nwin = a.n_save - a.win_begin;
                    a.median_scratch[(traj * count_median(a) + med) * nwin + (L.si - a.win_begin)] =
                        static_cast<float>(pick(v, a.feat_state[c]));
                    ++med;
                }
            }
            L.nsamp = n + 1;
        }
        if (a.y_full_out) {
            const int64_t base = ((int64_t)L.si * a.n_traj + traj) * S;
            if (a.y_out_dtype == PB_DTYPE_F64) {
                double* o = static_cast<double*>(a.y_full_out) + base;
#pragma unroll
                for (int s = 0; s < S; ++s) o[s] = static_cast<double>(v[s]);
            } else {
                float* o = static_cast<float*>(a.y_full_out) + base;
#pragma unroll
                for (int s = 0; s < S; ++s) o[s] = static_cast<float>(v[s]);
            }
        }
    }

    __device__ static int count_median(const pb_solve_args& a)
    {
        int m = 0;
        for (int c = 0; c < a.n_features; ++c) m += (a.feat_kind[c] == PB_FEAT_MEDIAN);
        return m;
    }

    // ---- start a trajectory: load y0/params, first derivative, initial step
    __device__ static void begin(L_t& L, int64_t traj, const pb_solve_args& a)
    {
        int64_t ic = traj, prow = 0;
        if (a.layout == PB_LAYOUT_CROSS) {
            ic = traj / a.n_param_rows;
            prow = traj - ic * a.n_param_rows;
        } else if (a.layout == PB_LAYOUT_INDEXED) {
            prow = __ldg(a.param_index + traj);
        }
        const bool bad_row = prow < 0 || prow >= a.n_param_rows;
        if (bad_row) prow = 0;
        double y0d[S];
#pragma unroll
        for (int s = 0; s < S; ++s) {
            y0d[s] = (a.y0_dtype == PB_DTYPE_F64) ? __ldg(static_cast<const double*>(a.y0) + ic * S + s)
                                                  : static_cast<double>(__ldg(static_cast<const float*>(a.y0) + ic * S + s));
            L.y[s] = static_cast<R>(y0d[s]);
            L.yc[s] = R(0);
        }
#pragma unroll
        for (int q = 0; q < Sys::NP; ++q)
            L.p[q] = q < a.n_params ? static_cast<R>(__ldg(a.params + prow * a.n_params + q)) : R(0);
        L.t = bad_row ? a.t1 : a.t0;  // a bad row finishes without stepping
        L.steps = 0;
        L.status = bad_row ? PB_TRAJ_BAD_INPUT : PB_TRAJ_OK;
        L.si = a.y_full_out ? 0 : a.win_begin;
        L.next_save = load_save(a, L.si);
        L.nsamp = 0;
        L.nan_mask = 0;
        L.cross_prev = 0;
#pragma unroll
        for (int s = 0; s < S; ++s) {
            L.shift[s] = 0.0;
            L.s1[s] = 0.0;
            L.s2[s] = 0.0;
            L.mn[s] = R(0);
            L.mx[s] = R(0);
            L.last[s] = R(0);
        }
#pragma unroll
        for (int j = 0; j < PB_MAX_CROSSING; ++j) L.cross_cnt[j] = 0;

        Sys::f(L.t, L.y, L.k1, L.p);
        // initial step size (dopri5_generic.zig:270-321); norms in FP64
        double d0 = 0.0, d1 = 0.0;
        double sc[S];
#pragma unroll
        for (int s = 0; s < S; ++s) {
            sc[s] = a.atol + fabs(y0d[s]) * a.rtol;
            const double r0 = y0d[s] / sc[s], r1 = static_cast<double>(L.k1[s]) / sc[s];
            d0 += r0 * r0;
            d1 += r1 * r1;
        }
        d0 = sqrt(d0 / S);
        d1 = sqrt(d1 / S);
        const double h0 = (d0 < 1e-5 || d1 < 1e-5) ? 1e-6 : 0.01 * d0 / d1;
        R ytmp[S], ftmp[S];
#pragma unroll
        for (int s = 0; s < S; ++s) ytmp[s] = static_cast<R>(y0d[s] + h0 * static_cast<double>(L.k1[s]));
        Sys::f(L.t + h0, ytmp, ftmp, L.p);
        double d2 = 0.0;
#pragma unroll
        for (int s = 0; s < S; ++s) {
            const double r = (static_cast<double>(ftmp[s]) - static_cast<double>(L.k1[s])) / sc[s];
            d2 += r * r;
        }
        d2 = sqrt(d2 / S) / h0;
        const double h1 = (d1 <= 1e-15 && d2 <= 1e-15) ? fmax(1e-6, h0 * 1e-3) : pow(0.01 / fmax(d1, d2), 0.2);
        L.dt = fmin(100.0 * h0, h1);
    }

    // ---- one attempted step; returns true once the trajectory is finished
    __device__ static bool step(L_t& L, int64_t traj, const pb_solve_args& a)
    {
        if (!(L.t < a.t1)) return true;
        if (L.steps >= a.max_steps) return true;
        L.steps++;
        double dt = L.dt;
        if (L.t + dt > a.t1) dt = a.t1 - L.t;
        if (dt <= 0.0) return true;
        if (L.t + dt == L.t) {
            L.status = PB_TRAJ_DT_UNDERFLOW;
            return true;
        }
        const R h = static_cast<R>(dt);
        const double t = L.t;
        R k2[S], k3[S], k4[S], k5[S], k6[S], k7[S], ys[S], d[S], yn[S];
#pragma unroll
        for (int s = 0; s < S; ++s) ys[s] = L.y[s] + h * (R(dp::a21) * L.k1[s]);
        Sys::f(t + dp::c2 * dt, ys, k2, L.p);
#pragma unroll
        for (int s = 0; s < S; ++s) ys[s] = L.y[s] + h * (R(dp::a31) * L.k1[s] + R(dp::a32) * k2[s]);
        Sys::f(t + dp::c3 * dt, ys, k3, L.p);
#pragma unroll
        for (int s = 0; s < S; ++s)
            ys[s] = L.y[s] + h * (R(dp::a41) * L.k1[s] + R(dp::a42) * k2[s] + R(dp::a43) * k3[s]);
        Sys::f(t + dp::c4 * dt, ys, k4, L.p);
#pragma unroll
        for (int s = 0; s < S; ++s)
            ys[s] = L.y[s] + h * (R(dp::a51) * L.k1[s] + R(dp::a52) * k2[s] + R(dp::a53) * k3[s] +
                                  R(dp::a54) * k4[s]);
        Sys::f(t + dp::c5 * dt, ys, k5, L.p);
#pragma unroll
        for (int s = 0; s < S; ++s)
            ys[s] = L.y[s] + h * (R(dp::a61) * L.k1[s] + R(dp::a62) * k2[s] + R(dp::a63) * k3[s] +
                                  R(dp::a64) * k4[s] + R(dp::a65) * k5[s]);
        Sys::f(t + dt, ys, k6, L.p);
#pragma unroll
        for (int s = 0; s < S; ++s) {
            d[s] = h * (R(dp::b1) * L.k1[s] + R(dp::b3) * k3[s] + R(dp::b4) * k4[s] + R(dp::b5) * k5[s] +
                        R(dp::b6) * k6[s]);
            yn[s] = L.y[s] + d[s];
        }
        Sys::f(t + dt, yn, k7, L.p);

        // embedded error estimate; the norm is accumulated in FP64
        double err = 0.0;
#pragma unroll
        for (int s = 0; s < S; ++s) {
            const R e = h * (R(dp::e1) * L.k1[s] + R(dp::e3) * k3[s] + R(dp::e4) * k4[s] + R(dp::e5) * k5[s] +
                             R(dp::e6) * k6[s] + R(dp::e7) * k7[s]);
            const double sc =
                a.atol + a.rtol * fmax(fabs(static_cast<double>(L.y[s])), fabs(static_cast<double>(yn[s])));
            const double r = static_cast<double>(e) / sc;
            err += r * r;
        }
        err = sqrt(err / S);
        if (!isfinite(err)) {
            L.status = PB_TRAJ_NONFINITE;
            return true;
        }

        const bool accept = err <= 1.0;
        if (accept) {
            const double tn = t + dt;
            if (L.next_save <= tn + dp::save_slack) {
                R ia[S], ib[S], icf[S];
#pragma unroll
                for (int s = 0; s < S; ++s) {
                    const R ym = L.y[s] + h * (R(dp::m1) * L.k1[s] + R(dp::m3) * k3[s] + R(dp::m4) * k4[s] +
                                               R(dp::m5) * k5[s] + R(dp::m6) * k6[s] + R(dp::m7) * k7[s]);
                    ia[s] = R(2) * h * (k7[s] - L.k1[s]) - R(8) * (yn[s] + L.y[s]) + R(16) * ym;
                    ib[s] = h * (R(5) * L.k1[s] - R(3) * k7[s]) + R(18) * L.y[s] + R(14) * yn[s] - R(32) * ym;
                    icf[s] = h * (k7[s] - R(4) * L.k1[s]) - R(11) * L.y[s] - R(5) * yn[s] + R(16) * ym;
                }
                while (L.si < a.n_save && L.next_save <= tn + dp::save_slack) {
                    R v[S];
                    if (L.next_save <= t + dp::save_slack) {
#pragma unroll
                        for (int s = 0; s < S; ++s) v[s] = L.y[s];
                    } else {
                        const R x = static_cast<R>((L.next_save - t) / dt);
#pragma unroll
                        for (int s = 0; s < S; ++s)
                            v[s] = L.y[s] + x * (h * L.k1[s] + x * (icf[s] + x * (ib[s] + x * ia[s])));
                    }
                    record(L, v, traj, a);
                    L.si++;
                    L.next_save = load_save(a, L.si);
                }
            }
            if (MIXED) {
                // compensated accumulation keeps the FP32 state from drifting over
                // ~1e4 accepted steps (Kahan summation of the increments d)
#pragma unroll
                for (int s = 0; s < S; ++s) {
                    const R corr = d[s] - L.yc[s];
                    const R ynew = L.y[s] + corr;
                    L.yc[s] = (ynew - L.y[s]) - corr;
                    L.y[s] = ynew;
                }
            } else {
#pragma unroll
                for (int s = 0; s < S; ++s) L.y[s] = yn[s];
            }
#pragma unroll
            for (int s = 0; s < S; ++s) L.k1[s] = k7[s];
            L.t = tn;
            if (a.unbounded_thr > 0.0) {
                double m = 0.0;
#pragma unroll
                for (int s = 0; s < S; ++s) m = fmax(m, fabs(static_cast<double>(L.y[s])));
                if (m >= a.unbounded_thr) {
                    L.status = PB_TRAJ_UNBOUNDED;
                    return true;
                }
            }
        }
        double fac;
        if (err == 0.0) {
            fac = dp::max_factor;
        } else {
            double g;
            if (MIXED) {
                g = static_cast<double>(0.9f * exp2f(-0.2f * log2f(static_cast<float>(err))));
            } else {
                g = dp::safety * pow(err, -0.2);
            }
            fac = fmin(dp::max_factor, fmax(accept ? 1.0 : dp::min_factor, g));
        }
        L.dt = dt * fac;
        return !(L.t < a.t1);
    }

    // ---- tail fill, features, status and states of a finished trajectory
    __device__ static void finish(L_t& L, int64_t traj, const pb_solve_args& a)
    {
        if (L.status == PB_TRAJ_OK && L.t < a.t1 && L.steps >= a.max_steps) L.status = PB_TRAJ_MAX_STEPS;
        R fill[S];
#pragma unroll
        for (int s = 0; s < S; ++s) fill[s] = (L.status == PB_TRAJ_UNBOUNDED) ? R(CUDART_INF) : L.y[s];
        while (L.si < a.n_save) {
            record(L, fill, traj, a);
            L.si++;
        }
        if (a.features_out) {
            const double n = static_cast<double>(L.nsamp);
            int j = 0;
            for (int c = 0; c < a.n_features; ++c) {
                const int kind = a.feat_kind[c];
                const int st = a.feat_state[c];
                const double sh = pick(L.shift, st), s1 = pick(L.s1, st), s2 = pick(L.s2, st);
                const bool has_nan = (L.nan_mask >> st) & 1u;
                double mx = has_nan ? CUDART_NAN : static_cast<double>(pick(L.mx, st));
                double mn = has_nan ? CUDART_NAN : static_cast<double>(pick(L.mn, st));
                const double mean = sh + s1 / n;
                const double var = fmax((s2 - s1 * (s1 / n)) / n, 0.0);
                double v;
                switch (kind) {
                    case PB_FEAT_MEAN: v = mean; break;
                    case PB_FEAT_STD: v = sqrt(var); break;
                    case PB_FEAT_VAR: v = var; break;
                    case PB_FEAT_RMS: v = sqrt((s2 + sh * (2.0 * s1 + n * sh)) / n); break;
                    case PB_FEAT_MAX: v = mx; break;
                    case PB_FEAT_ABSMAX: v = fmax(fabs(mx), fabs(mn)); break;
                    case PB_FEAT_MIN: v = mn; break;
                    case PB_FEAT_DELTA: v = fabs(mx - mean); break;
                    case PB_FEAT_LOG_DELTA: v = log(fabs(mx - mean) + 1e-10); break;
                    case PB_FEAT_AMPLITUDE: v = mx - mn; break;
                    case PB_FEAT_CROSSINGS:
                        v = (j < PB_MAX_CROSSING) ? static_cast<double>(pick(L.cross_cnt, j)) : CUDART_NAN;
                        ++j;
                        break;
                    case PB_FEAT_LAST: v = static_cast<double>(pick(L.last, st)); break;
                    case PB_FEAT_MEDIAN: continue;  // written by the median pass
                    default: v = CUDART_NAN;
                }
                if (L.nsamp == 0) v = CUDART_NAN;
                a.features_out[traj * a.n_features + c] = v;
            }
        }
        if (a.status_out) a.status_out[traj] = L.status;
        if (a.steps_out) a.steps_out[traj] = L.steps;
        if (a.y_final_out) {
            if (a.y_out_dtype == PB_DTYPE_F64) {
                double* o = static_cast<double*>(a.y_final_out) + traj * S;
#pragma unroll
                for (int s = 0; s < S; ++s) o[s] = static_cast<double>(L.y[s]);
            } else {
                float* o = static_cast<float*>(a.y_final_out) + traj * S;
#pragma unroll
                for (int s = 0; s < S; ++s) o[s] = static_cast<float>(L.y[s]);
            }
        }
    }
};

// Warp-aggregated fetch from the global work queue: one atomicAdd per warp for
// all lanes in `mask`; returns this lane's trajectory index (valid if in mask).
__device__ __forceinline__ int64_t warp_fetch(unsigned long long* q, unsigned mask, int lane)
{
    const int leader = __ffs(mask) - 1;
    unsigned long long base = 0;
    if (lane == leader) base = atomicAdd(q, static_cast<unsigned long long>(__popc(mask)));
    base = __shfl_sync(mask, base, leader);
    const int rank = __popc(mask & ((1u << lane) - 1u));
    return static_cast<int64_t>(base) + rank;
}

// Plain schedule: one thread per trajectory, no queue (the FP64 baseline K1
// when R = double).
template <class Sys, class R, bool MIXED>
__global__ void __launch_bounds__(256) k_solve_plain(const pb_solve_args a)
{
    using I = Integrator<Sys, R, MIXED>;
    const int64_t traj = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (traj >= a.n_traj) return;
    typename I::L_t L;
    I::begin(L, traj, a);
    while (!I::step(L, traj, a)) {
    }
    I::finish(L, traj, a);
}

// Queue schedule: persistent lanes; a lane whose trajectory finished takes the
// next one from the global queue (warp-aggregated), so long trajectories do not
// leave the rest of their warp idle.  Every loop is bounded: each trajectory
// runs at most max_steps attempted steps and the queue holds n_traj entries.
template <class Sys, class R, bool MIXED>
__global__ void __launch_bounds__(256) k_solve_queue(const pb_solve_args a)
{
    using I = Integrator<Sys, R, MIXED>;
    const int lane = threadIdx.x & 31;
    typename I::L_t L;
    int64_t traj = warp_fetch(a.queue_counter, 0xffffffffu, lane);
    bool have = traj < a.n_traj;
    bool exhausted = !have;
    if (have) I::begin(L, traj, a);
    while (__any_sync(0xffffffffu, have)) {
        if (have && I::step(L, traj, a)) {
            I::finish(L, traj, a);
            have = false;
        }
        const bool want = !have && !exhausted;
        const unsigned m = __ballot_sync(0xffffffffu, want);
        if (m) {
            if (want) {
                const int64_t nt = warp_fetch(a.queue_counter, m, lane);
                if (nt < a.n_traj) {
                    traj = nt;
                    have = true;
                    I::begin(L, traj, a);
                } else {
                    exhausted = true;
                }
            }
        }
    }
}

}  // namespace pb
