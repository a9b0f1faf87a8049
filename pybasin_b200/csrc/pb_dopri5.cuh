// Per-lane adaptive Dormand-Prince 5(4) integrator with dense output fused
// into streaming window statistics.
//
// One CUDA thread owns one trajectory at a time; its state and stages live in
// registers, its window statistics in a per-thread slot of shared memory (they
// are touched only at save points, so keeping them out of the register file
// lets every trajectory of a 100k-IC batch be resident at once).  The algorithm
// (tableau, Shampine error estimate, torchdiffeq-style control, 4th-order dense
// output) is the reference's native solver,
// src/zigode/src/solver/dopri5_generic.zig:
//   step and stages      :130-183
//   RMS error norm       :185-192
//   dense output         :194-221
//   FSAL swap            :223-225
//   step-size control    :228-235 (safety 0.9, min 0.2, max 10, no shrink on accept)
//   initial step size    :270-321 (Hairer, Norsett & Wanner II.4)
//   tail fill            :238-241
// Statistics follow src/pybasin/ts_torch/calculators/torch_features_statistical.py
// (:30-110, :307-318) and torch_features_pattern.py:56-60, as streaming
// shifted-sum reductions over the save points of the window.
//
// Precision: Integrator<Sys, double> is the plain FP64 kernel (every operation
// in FP64, control identical to the reference).  Integrator<Sys, float> runs
// stages, state and dense output in FP32 (state increments Kahan-compensated),
// keeps time, step size and the error-norm accumulation in FP64, and evaluates
// the step-size factor in FP32.
#pragma once

#include "pb_compat.cuh"
#include "pb_rhs.cuh"
#include "pb_scratch.cuh"
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

// Block-wide plan derived once from the arguments (shared memory).
struct Plan {
    int n_cross;
    int n_med;
    unsigned stat_mask;  // states that any feature column reads
    int ns;              // number of such states ("slots", in state order)
    int stat_state[PB_MAX_STAT_STATES];
    int slot_of[PB_MAX_STAT_STATES];
    int cross_state[PB_MAX_CROSSING];
    double cross_level[PB_MAX_CROSSING];
    int med_state[PB_MAX_FEATURES];
    ScratchLayout sl;
    double inv_ds;  // 1 / mean spacing of the save grid (a hint for locating save points)
};

__device__ __forceinline__ void build_plan(Plan& pl, const pb_solve_args& a)
{
    int nc = 0, nm = 0;
    unsigned mask = 0;
    for (int c = 0; c < a.n_features; ++c) {
        mask |= 1u << a.feat_state[c];
        if (a.feat_kind[c] == PB_FEAT_CROSSINGS && nc < PB_MAX_CROSSING) {
            pl.cross_state[nc] = a.feat_state[c];
            pl.cross_level[nc] = a.feat_param[c];
            ++nc;
        } else if (PB_FEAT_IS_WINDOW(a.feat_kind[c])) {
            pl.med_state[nm++] = a.feat_state[c];
        }
    }
    pl.n_cross = nc;
    pl.n_med = nm;
    pl.stat_mask = mask;
    int ns = 0;
    for (int st = 0; st < PB_MAX_STAT_STATES; ++st) {
        pl.slot_of[st] = -1;
        if ((mask >> st) & 1u) {
            pl.slot_of[st] = ns;
            pl.stat_state[ns++] = st;
        }
    }
    pl.ns = ns;
    for (int j = ns; j < PB_MAX_STAT_STATES; ++j) pl.stat_state[j] = 0;  // unused slots read state 0
    pl.sl = scratch_layout(a);
    pl.inv_ds = (a.n_save > 1 && a.save_ts[a.n_save - 1] > a.save_ts[0])
                    ? (a.n_save - 1) / (a.save_ts[a.n_save - 1] - a.save_ts[0])
                    : 0.0;
}

// Per-thread window statistics in shared memory, structure-of-arrays
// (consecutive threads hit consecutive words).  Layout of the dynamic segment:
//   double [6*S][nthr]: shift, s1, s2, min, max, last (per state)
//   int    [PB_MAX_CROSSING + 2][nthr]: crossing counts, nsamp, flags
// flags: bits 0..7 = NaN seen per state, bits 8..11 = previous sample above level.
template <int S>
struct Stats {
    double* d;
    int* i;
    int nthr, tid;
    static constexpr int kBytesPerThread = 6 * S * 8 + (PB_MAX_CROSSING + 2) * 4;
    __device__ __forceinline__ double& shift(int s) { return d[(0 * S + s) * nthr + tid]; }
    __device__ __forceinline__ double& s1(int s) { return d[(1 * S + s) * nthr + tid]; }
    __device__ __forceinline__ double& s2(int s) { return d[(2 * S + s) * nthr + tid]; }
    __device__ __forceinline__ double& mn(int s) { return d[(3 * S + s) * nthr + tid]; }
    __device__ __forceinline__ double& mx(int s) { return d[(4 * S + s) * nthr + tid]; }
    __device__ __forceinline__ double& last(int s) { return d[(5 * S + s) * nthr + tid]; }
    __device__ __forceinline__ int& cross(int j) { return i[j * nthr + tid]; }
    __device__ __forceinline__ int& nsamp() { return i[PB_MAX_CROSSING * nthr + tid]; }
    __device__ __forceinline__ int& flags() { return i[(PB_MAX_CROSSING + 1) * nthr + tid]; }
    __device__ __forceinline__ void reset()
    {
#pragma unroll
        for (int s = 0; s < S; ++s) {
            shift(s) = 0.0;
            s1(s) = 0.0;
            s2(s) = 0.0;
            mn(s) = CUDART_INF;
            mx(s) = -CUDART_INF;
            last(s) = 0.0;
        }
#pragma unroll
        for (int j = 0; j < PB_MAX_CROSSING; ++j) cross(j) = 0;
        nsamp() = 0;
        flags() = 0;
    }
};

template <class Sys, class R>
struct Lane {
    static constexpr int S = Sys::S;
    R y[S];
    R yc[S];  // Kahan compensation of y (FP32 kernel only)
    R k1[S];
    R p[Sys::NP];
    double t, dt;
    double next_save;  // save_ts[si] (or +inf past the end)
    float phase;       // FP32 clock: t mod 2 pi of the current t (kept across steps)
    int si;            // next save index
    int steps;
    int max_steps;     // a.max_steps clamped to int range (a 32-bit compare per step)
    int status;
    int nrec;          // deferred dense output: records written (-1 = capacity exceeded)
};

// 2^x by the hardware approximation (ex2.approx.ftz.f32, relative error ~2^-22):
// ample for a step-size factor that is clamped to [0.2, 10] afterwards
__device__ __forceinline__ float ex2_approx(float x)
{
    float r;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

__device__ __forceinline__ double load_save(const pb_solve_args& a, int si)
{
    return si < a.n_save ? __ldg(a.save_ts + si) : CUDART_INF;
}

template <class Sys, class R>
struct Integrator {
    static constexpr int S = Sys::S;
    static constexpr bool MIXED = same_type<R, float>::value;
    // FP32 phase clock (t mod 2 pi) for the built-in periodically forced systems;
    // a system that declares kExactTime gets t in FP64 at every stage instead
    static constexpr bool F32_CLOCK = MIXED && !exact_time<Sys>::value;
    using L_t = Lane<Sys, R>;
    using St = Stats<S>;

    // ---- the save points inside (t, tn]: interpolate each (`interp` produces the
    // sample at save instant ts) and fold it into register partials of the window
    // statistics, merged into the shared-memory slot once per run.  The next save
    // instant is fetched one iteration ahead so its load latency overlaps the work.
    template <class Interp>
    __device__ static void record_run(L_t& L, St& st, const Plan& pl, int64_t traj, const pb_solve_args& a,
                                      double tn, const Interp& interp)
    {
        const bool stats_on = pl.stat_mask != 0;
        const int64_t nwin = a.n_save - a.win_begin;
        const int n = st.nsamp();
        int flg = st.flags();
        R sh[S], ls1[S], ls2[S], lmn[S], lmx[S], llast[S];
#pragma unroll
        for (int s = 0; s < S; ++s) {
            sh[s] = static_cast<R>(st.shift(s));
            ls1[s] = R(0);
            ls2[s] = R(0);
            lmn[s] = R(CUDART_INF);
            lmx[s] = R(-CUDART_INF);
            llast[s] = R(0);
        }
        int cnt = 0;
        double ts = L.next_save;
        while (L.si < a.n_save && ts <= tn + dp::save_slack) {
            const double ts_next = load_save(a, L.si + 1);
            R v[S];
            interp(ts, v);
            if (L.si >= a.win_begin && stats_on) {
                const bool first = (n + cnt) == 0;
#pragma unroll
                for (int s = 0; s < S; ++s) {
                    if (!((pl.stat_mask >> s) & 1)) continue;
                    if (first) sh[s] = isfinite(v[s]) ? v[s] : R(0);
                    const R dd = v[s] - sh[s];
                    ls1[s] += dd;
                    ls2[s] = fma(dd, dd, ls2[s]);
                    lmn[s] = fmin(lmn[s], v[s]);
                    lmx[s] = fmax(lmx[s], v[s]);
                    llast[s] = v[s];
                    if (v[s] != v[s]) flg |= 1 << s;
                }
                for (int j = 0; j < pl.n_cross; ++j) {
                    const bool above = static_cast<double>(pick(v, pl.cross_state[j])) > pl.cross_level[j];
                    const bool prev = (flg >> (8 + j)) & 1;
                    if (!first && above != prev) st.cross(j) += 1;
                    flg = (flg & ~(1 << (8 + j))) | (static_cast<int>(above) << (8 + j));
                }
                for (int m = 0; m < pl.n_med; ++m)
                    median_ptr(a, pl.sl)[(traj * pl.n_med + m) * nwin + (L.si - a.win_begin)] =
                        static_cast<float>(pick(v, pl.med_state[m]));
                ++cnt;
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
            L.si++;
            ts = ts_next;
        }
        L.next_save = ts;
        if (cnt > 0) {
#pragma unroll
            for (int s = 0; s < S; ++s) {
                if (!((pl.stat_mask >> s) & 1)) continue;
                if (n == 0) st.shift(s) = static_cast<double>(sh[s]);
                st.s1(s) += static_cast<double>(ls1[s]);
                st.s2(s) += static_cast<double>(ls2[s]);
                st.mn(s) = fmin(st.mn(s), static_cast<double>(lmn[s]));
                st.mx(s) = fmax(st.mx(s), static_cast<double>(lmx[s]));
                st.last(s) = static_cast<double>(llast[s]);
            }
            st.nsamp() = n + cnt;
            st.flags() = flg;
        }
    }

    // ---- start a trajectory: load y0/params, first derivative, initial step
    // (y0 row, parameter row) of a trajectory; false for a parameter row out of range
    __device__ static bool rows_of(int64_t traj, const pb_solve_args& a, int64_t& ic, int64_t& prow)
    {
        ic = traj;
        prow = 0;
        if (a.layout == PB_LAYOUT_CROSS) {
            ic = traj / a.n_param_rows;
            prow = traj - ic * a.n_param_rows;
        } else if (a.layout == PB_LAYOUT_INDEXED) {
            prow = __ldg(a.param_index + traj);
        }
        const bool bad_row = prow < 0 || prow >= a.n_param_rows;
        if (bad_row) prow = 0;
        return !bad_row;
    }

    __device__ static void load_params(L_t& L, int64_t prow, const pb_solve_args& a)
    {
#pragma unroll
        for (int q = 0; q < Sys::NP; ++q)
            L.p[q] = q < a.n_params ? static_cast<R>(__ldg(a.params + prow * a.n_params + q)) : R(0);
    }

    // ---- probed schedule: the state after the probe phase, and back
    __device__ static void save(const L_t& L, const Plan& pl, int64_t traj, const pb_solve_args& a, int done)
    {
        unsigned char* b = state_ptr(a, pl.sl, traj);
        R* r = reinterpret_cast<R*>(b);
#pragma unroll
        for (int s = 0; s < S; ++s) {
            r[s] = L.y[s];
            r[S + s] = L.yc[s];
            r[2 * S + s] = L.k1[s];
        }
        double* d = reinterpret_cast<double*>(b + (3 * S * sizeof(R) + 7) / 8 * 8);
        d[0] = L.t;
        d[1] = L.dt;
        d[2] = L.next_save;
        int* i = reinterpret_cast<int*>(d + 3);
        i[0] = L.si;
        i[1] = L.steps;
        i[2] = L.status;
        i[3] = L.nrec;
        i[4] = done;
    }

    // false if the trajectory already finished in the probe phase
    __device__ static bool resume(L_t& L, const Plan& pl, int64_t traj, const pb_solve_args& a)
    {
        const unsigned char* b = state_ptr(a, pl.sl, traj);
        const double* d = reinterpret_cast<const double*>(b + (3 * S * sizeof(R) + 7) / 8 * 8);
        const int* i = reinterpret_cast<const int*>(d + 3);
        if (i[4]) return false;
        const R* r = reinterpret_cast<const R*>(b);
#pragma unroll
        for (int s = 0; s < S; ++s) {
            L.y[s] = r[s];
            L.yc[s] = r[S + s];
            L.k1[s] = r[2 * S + s];
        }
        L.t = d[0];
        L.dt = d[1];
        L.next_save = d[2];
        L.si = i[0];
        L.steps = i[1];
        L.status = i[2];
        L.nrec = i[3];
        L.phase = (F32_CLOCK && Sys::kTime) ? reduce_two_pi(L.t) : 0.f;
        L.max_steps = static_cast<int>(a.max_steps < 0x7fffffffLL ? a.max_steps : 0x7fffffffLL);
        int64_t ic, prow;
        rows_of(traj, a, ic, prow);
        load_params(L, prow, a);
        return true;
    }

    __device__ static void begin(L_t& L, St& st, int64_t traj, const pb_solve_args& a)
    {
        int64_t ic, prow;
        const bool bad_row = !rows_of(traj, a, ic, prow);
        double y0d[S];
#pragma unroll
        for (int s = 0; s < S; ++s) {
            y0d[s] = (a.y0_dtype == PB_DTYPE_F64)
                         ? __ldg(static_cast<const double*>(a.y0) + ic * S + s)
                         : static_cast<double>(__ldg(static_cast<const float*>(a.y0) + ic * S + s));
            L.y[s] = static_cast<R>(y0d[s]);
            L.yc[s] = R(0);
        }
        load_params(L, prow, a);
        L.t = bad_row ? a.t1 : a.t0;  // a bad row finishes without stepping
        L.steps = 0;
        L.max_steps = static_cast<int>(a.max_steps < 0x7fffffffLL ? a.max_steps : 0x7fffffffLL);
        L.status = bad_row ? PB_TRAJ_BAD_INPUT : PB_TRAJ_OK;
        L.si = a.y_full_out ? 0 : a.win_begin;
        L.next_save = load_save(a, L.si);
        L.nrec = 0;
        L.phase = (F32_CLOCK && Sys::kTime) ? reduce_two_pi(L.t) : 0.f;
        if (st.d) st.reset();

        // first derivative and initial step size (dopri5_generic.zig:270-321), norms in FP64
        if constexpr (F32_CLOCK) {
            Sys::f(ClockF32{reduce_two_pi(a.t0)}, L.y, L.k1, L.p);
        } else {
            Sys::f(ClockF64{a.t0}, L.y, L.k1, L.p);
        }
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
        if constexpr (F32_CLOCK) {
            Sys::f(ClockF32{reduce_two_pi(a.t0 + h0)}, ytmp, ftmp, L.p);
        } else {
            Sys::f(ClockF64{a.t0 + h0}, ytmp, ftmp, L.p);
        }
        double d2 = 0.0;
#pragma unroll
        for (int s = 0; s < S; ++s) {
            const double r = (static_cast<double>(ftmp[s]) - static_cast<double>(L.k1[s])) / sc[s];
            d2 += r * r;
        }
        d2 = sqrt(d2 / S) / h0;
        const double h1 =
            (d1 <= 1e-15 && d2 <= 1e-15) ? fmax(1e-6, h0 * 1e-3) : pow(0.01 / fmax(d1, d2), 0.2);
        L.dt = fmin(100.0 * h0, h1);
    }

    // ---- deferred dense output: one record per accepted window step holding save
    // points (step start, step size, first covered save, count, and for each
    // statistics state y, h*k1 and the three higher polynomial coefficients)
    __device__ static bool write_record(L_t& L, const Plan& pl, int64_t traj, const pb_solve_args& a, double t,
                                        double dt, R h, const R (&ia)[S], const R (&ib)[S], const R (&icf)[S],
                                        double tn)
    {
        if (L.nrec >= pl.sl.cap) return false;
        // first save index after (t, tn]: probe where a uniform grid would put it,
        // then correct (the grid is not assumed uniform, only used as a hint)
        const double lim = tn + dp::save_slack;
        int si;
        double ts;
        {
            const int guess = min(L.si + 1 + static_cast<int>(fmax(0.0, (lim - L.next_save) * pl.inv_ds)), a.n_save);
            // both neighbours of the guess in one round trip; exact for a uniform grid
            const double below = guess > L.si + 1 ? load_save(a, guess - 1) : L.next_save;
            const double above = load_save(a, guess);
            if (below <= lim && !(above <= lim)) {
                si = guess;
                ts = above;
            } else {
                int g = guess;
                while (g > L.si + 1 && !(load_save(a, g - 1) <= lim)) --g;  // move down to a covered index
                while (g < a.n_save && load_save(a, g) <= lim) ++g;         // move up past the covered run
                si = g;
                ts = load_save(a, si);
            }
        }
        unsigned char* rec = record_ptr(a, pl.sl, traj, L.nrec);
        if constexpr (S <= 4) {
            // every word at a compile-time position: slot j holds state stat_state[j]
            // (picked by value), slots past ns land in padding or past the stride;
            // then 16-byte vector stores of the record's stride
            constexpr int RW = sizeof(R) / 4;
            constexpr int kWords = (kRecordHeader + 5 * S * static_cast<int>(sizeof(R)) + 15) / 16 * 4;
            unsigned w[kWords];
#pragma unroll
            for (int q = 0; q < kWords; ++q) w[q] = 0u;
            w[0] = __double2loint(t);
            w[1] = __double2hiint(t);
            w[2] = __double2loint(dt);
            w[3] = __double2hiint(dt);
            w[kRecordIndexOffset / 4] = static_cast<unsigned>(L.si);
            w[kRecordIndexOffset / 4 + 1] = static_cast<unsigned>(si - L.si);
#pragma unroll
            for (int j = 0; j < S; ++j) {
                const int s = pl.stat_state[j];
                const R vals[5] = {pick(L.y, s), h * pick(L.k1, s), pick(icf, s), pick(ib, s), pick(ia, s)};
#pragma unroll
                for (int q = 0; q < 5; ++q) {
                    const int base = kRecordHeader / 4 + (5 * j + q) * RW;
                    if constexpr (RW == 1) {
                        w[base] = __float_as_uint(static_cast<float>(vals[q]));
                    } else {
                        const double dv = static_cast<double>(vals[q]);
                        w[base] = static_cast<unsigned>(__double2loint(dv));
                        w[base + 1] = static_cast<unsigned>(__double2hiint(dv));
                    }
                }
            }
            uint4* dst = reinterpret_cast<uint4*>(rec);
            const int n16 = pl.sl.rec_stride / 16;
#pragma unroll
            for (int z = 0; z < kWords / 4; ++z)
                if (z < n16) dst[z] = make_uint4(w[4 * z], w[4 * z + 1], w[4 * z + 2], w[4 * z + 3]);
        } else {
            // wider systems: scalar stores of the statistics states only
            double* hd = reinterpret_cast<double*>(rec);
            hd[0] = t;
            hd[1] = dt;
            reinterpret_cast<int2*>(rec + kRecordIndexOffset)[0] = make_int2(L.si, si - L.si);
            R* c = reinterpret_cast<R*>(rec + kRecordHeader);
#pragma unroll
            for (int s = 0; s < S; ++s) {
                if (!((pl.stat_mask >> s) & 1u)) continue;
                c[0] = L.y[s];
                c[1] = h * L.k1[s];
                c[2] = icf[s];
                c[3] = ib[s];
                c[4] = ia[s];
                c += 5;
            }
        }
        L.si = si;
        L.next_save = ts;
        L.nrec++;
        return true;
    }

    template <class TB>
    __device__ __forceinline__ static void stages(const TB& tb, const L_t& L, R h, R (&k2)[S], R (&k3)[S],
                                                  R (&k4)[S], R (&k5)[S], R (&k6)[S], R (&k7)[S], R (&d)[S],
                                                  R (&yn)[S])
    {
        // stage arguments y + h * sum_j a_ij k_j, the sum accumulated oldest stage
        // first (the newest stage enters the last multiply-add)
        R ys[S];
#pragma unroll
        for (int s = 0; s < S; ++s) ys[s] = fmad(h, R(dp::a21) * L.k1[s], L.y[s]);
        Sys::f(tb.at(dp::c2), ys, k2, L.p);
#pragma unroll
        for (int s = 0; s < S; ++s) ys[s] = fmad(h, fmad(R(dp::a32), k2[s], R(dp::a31) * L.k1[s]), L.y[s]);
        Sys::f(tb.at(dp::c3), ys, k3, L.p);
#pragma unroll
        for (int s = 0; s < S; ++s)
            ys[s] = fmad(h, fmad(R(dp::a43), k3[s], fmad(R(dp::a42), k2[s], R(dp::a41) * L.k1[s])), L.y[s]);
        Sys::f(tb.at(dp::c4), ys, k4, L.p);
#pragma unroll
        for (int s = 0; s < S; ++s)
            ys[s] = fmad(h,
                         fmad(R(dp::a54), k4[s],
                              fmad(R(dp::a53), k3[s], fmad(R(dp::a52), k2[s], R(dp::a51) * L.k1[s]))),
                         L.y[s]);
        Sys::f(tb.at(dp::c5), ys, k5, L.p);
#pragma unroll
        for (int s = 0; s < S; ++s)
            ys[s] = fmad(h,
                         fmad(R(dp::a65), k5[s],
                              fmad(R(dp::a64), k4[s],
                                   fmad(R(dp::a63), k3[s], fmad(R(dp::a62), k2[s], R(dp::a61) * L.k1[s])))),
                         L.y[s]);
        Sys::f(tb.at(1.0), ys, k6, L.p);
#pragma unroll
        for (int s = 0; s < S; ++s) {
            d[s] = h * fmad(R(dp::b6), k6[s],
                            fmad(R(dp::b5), k5[s], fmad(R(dp::b4), k4[s], fmad(R(dp::b3), k3[s], R(dp::b1) * L.k1[s]))));
            yn[s] = L.y[s] + d[s];
        }
        Sys::f(tb.at(1.0), yn, k7, L.p);
    }

    // h * sum_j e_j k_j, the embedded error estimate of one state
    __device__ __forceinline__ static R err_est(R h, R k1, R k3, R k4, R k5, R k6, R k7)
    {
        return h * fmad(R(dp::e7), k7,
                        fmad(R(dp::e6), k6, fmad(R(dp::e5), k5, fmad(R(dp::e4), k4, fmad(R(dp::e3), k3, R(dp::e1) * k1)))));
    }

    // ---- one attempted step; returns true once the trajectory is finished
    template <bool DEFER>
    __device__ static bool step(L_t& L, St& st, const Plan& pl, int64_t traj, const pb_solve_args& a)
    {
        if (!(L.t < a.t1) || L.steps >= L.max_steps) return true;
        L.steps++;
        const double t = L.t;
        // the stage phase base of t was reduced during the previous step (from its
        // end point, known as soon as its dt was), off this step's dependency chain
        const float r0 = L.phase;
        double dt = L.dt;
        R h = static_cast<R>(dt);
        if (t + dt > a.t1) {
            dt = a.t1 - t;
            h = static_cast<R>(dt);
        }
        // dt > 0 here (t < t1, and the control keeps dt * fac with fac >= 0.2);
        // a dt lost below t's resolution (including 0) ends the trajectory
        if (t + dt == t) {
            L.status = PB_TRAJ_DT_UNDERFLOW;
            return true;
        }
        R k2[S], k3[S], k4[S], k5[S], k6[S], k7[S], d[S], yn[S];
        if constexpr (F32_CLOCK) {
            stages(TimeBaseF32{r0, static_cast<float>(h)}, L, h, k2, k3, k4, k5, k6, k7, d, yn);
        } else {
            stages(TimeBaseF64{t, dt}, L, h, k2, k3, k4, k5, k6, k7, d, yn);
        }

        // embedded error estimate (RMS norm, dopri5_generic.zig:185-192)
        double err2 = 0.0;
        float e2f = 0.f;  // the same sum in FP32, feeding only the step-size factor
        if (MIXED) {
            const float rt = static_cast<float>(a.rtol), at = static_cast<float>(a.atol);
#pragma unroll
            for (int s = 0; s < S; ++s) {
                const float e = static_cast<float>(err_est(h, L.k1[s], k3[s], k4[s], k5[s], k6[s], k7[s]));
                const float sc =
                    fmaf(rt, fmaxf(fabsf(static_cast<float>(L.y[s])), fabsf(static_cast<float>(yn[s]))), at);
                const float rf = __fdividef(e, sc);
                const double r = static_cast<double>(rf);
                err2 = fma(r, r, err2);
                e2f = fmaf(rf, rf, e2f);
            }
            err2 *= 1.0 / S;
            e2f *= 1.f / S;
        } else {
#pragma unroll
            for (int s = 0; s < S; ++s) {
                const double e = static_cast<double>(err_est(h, L.k1[s], k3[s], k4[s], k5[s], k6[s], k7[s]));
                const double sc =
                    a.atol + a.rtol * fmax(fabs(static_cast<double>(L.y[s])), fabs(static_cast<double>(yn[s])));
                const double r = e / sc;
                err2 += r * r;
            }
            err2 /= S;
        }
        if (!isfinite(err2)) {
            L.status = PB_TRAJ_NONFINITE;
            return true;
        }
        const bool accept = err2 <= 1.0;
        const double tn = t + dt;
        // phase base for the next step if this one is accepted (depends on t and dt only)
        const float phase_next = (F32_CLOCK && Sys::kTime) ? reduce_two_pi(tn) : 0.f;

        if (accept && L.next_save <= tn + dp::save_slack) {
            // dense output (dopri5_generic.zig:194-221): 4th-order polynomial in x = (ts - t)/dt
            R ia[S], ib[S], icf[S];
#pragma unroll
            for (int s = 0; s < S; ++s) {
                const R ym = fmad(
                    h,
                    fmad(R(dp::m7), k7[s],
                         fmad(R(dp::m6), k6[s],
                              fmad(R(dp::m5), k5[s], fmad(R(dp::m4), k4[s], fmad(R(dp::m3), k3[s], R(dp::m1) * L.k1[s]))))),
                    L.y[s]);
                ia[s] = fmad(R(16), ym, fmad(R(-8), yn[s] + L.y[s], (R(2) * h) * (k7[s] - L.k1[s])));
                ib[s] = fmad(R(-32), ym, fmad(R(14), yn[s], fmad(R(18), L.y[s], h * fmad(R(5), L.k1[s], R(-3) * k7[s]))));
                icf[s] = fmad(R(16), ym, fmad(R(-5), yn[s], fmad(R(-11), L.y[s], h * fmad(R(-4), L.k1[s], k7[s]))));
            }
            if (DEFER) {
                if (!write_record(L, pl, traj, a, t, dt, h, ia, ib, icf, tn)) {
                    L.nrec = -1;  // capacity exceeded: the inline pass integrates it again
                    return true;
                }
            } else {
            const double inv_dt = 1.0 / dt;
            record_run(L, st, pl, traj, a, tn, [&](double ts, R (&v)[S]) {
                if (ts <= t + dp::save_slack) {
#pragma unroll
                    for (int s = 0; s < S; ++s) v[s] = L.y[s];
                } else {
                    const R x = static_cast<R>((ts - t) * inv_dt);
#pragma unroll
                    for (int s = 0; s < S; ++s)
                        v[s] = fmad(x, fmad(x, fmad(x, fmad(x, ia[s], ib[s]), icf[s]), h * L.k1[s]), L.y[s]);
                }
            });
            }
        }
        if (accept) {
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
            L.phase = phase_next;
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
        // step-size control (dopri5_generic.zig:228-235)
        double fac;
        if (MIXED) {
            // acceptance above used the FP64 norm; the factor 0.9 * err^-0.2 needs no
            // more than FP32, and taking it from the FP32 sum keeps the FP64
            // conversions off the step-to-step dependency chain
            const float g = 0.9f * ex2_approx(-0.1f * __log2f(e2f));
            fac = (e2f == 0.f) ? dp::max_factor : static_cast<double>(fminf(10.f, fmaxf(accept ? 1.f : 0.2f, g)));
        } else {
            const double err = sqrt(err2);
            fac = (err == 0.0) ? dp::max_factor
                               : fmin(dp::max_factor, fmax(accept ? 1.0 : dp::min_factor, dp::safety * pow(err, -0.2)));
        }
        L.dt = dt * fac;
        return !(L.t < a.t1);
    }

    // ---- tail fill, features, status and states of a finished trajectory
    template <bool DEFER>
    __device__ static void finish(L_t& L, St& st, const Plan& pl, int64_t traj, const pb_solve_args& a)
    {
        if (L.status == PB_TRAJ_OK && L.t < a.t1 && L.steps >= L.max_steps) L.status = PB_TRAJ_MAX_STEPS;
        if (DEFER) {
            // the sampling pass evaluates the records and fills the uncovered tail
            unsigned char* tl = tail_ptr(a, pl.sl, traj);
            int* ti = reinterpret_cast<int*>(tl);
            ti[0] = L.nrec;
            ti[1] = L.si;
            ti[2] = L.status;
            double* fillv = reinterpret_cast<double*>(tl + 16);
#pragma unroll
            for (int s = 0; s < S; ++s)
                fillv[s] = (L.status == PB_TRAJ_UNBOUNDED) ? CUDART_INF : static_cast<double>(L.y[s]);
            if (L.nrec < 0) return;  // the inline pass writes this trajectory's outputs
        } else {
        R fill[S];
#pragma unroll
        for (int s = 0; s < S; ++s) fill[s] = (L.status == PB_TRAJ_UNBOUNDED) ? R(CUDART_INF) : L.y[s];
        record_run(L, st, pl, traj, a, CUDART_INF, [&](double, R (&v)[S]) {
#pragma unroll
            for (int s = 0; s < S; ++s) v[s] = fill[s];
        });
        if (a.features_out) {
            const int ns = st.nsamp();
            const double n = static_cast<double>(ns);
            const int flg = st.flags();
            int j = 0;
            for (int c = 0; c < a.n_features; ++c) {
                const int kind = a.feat_kind[c];
                const int sidx = a.feat_state[c];
                const double sh = st.shift(sidx), s1 = st.s1(sidx), s2 = st.s2(sidx);
                const bool has_nan = (flg >> sidx) & 1;
                const double mx = has_nan ? CUDART_NAN : st.mx(sidx);
                const double mn = has_nan ? CUDART_NAN : st.mn(sidx);
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
                        v = (j < pl.n_cross) ? static_cast<double>(st.cross(j)) : CUDART_NAN;
                        ++j;
                        break;
                    case PB_FEAT_LAST: v = st.last(sidx); break;
                    case PB_FEAT_SUM: v = n * sh + s1; break;
                    case PB_FEAT_ABS_ENERGY: v = s2 + sh * (2.0 * s1 + n * sh); break;
                    case PB_FEAT_LENGTH: v = n; break;
                    case PB_FEAT_VARIATION_COEFF: v = sqrt(var) / (fabs(mean) + 1e-10); break;
                    default:
                        if (PB_FEAT_IS_WINDOW(kind)) continue;  // written by the window pass
                        v = CUDART_NAN;
                }
                if (ns == 0) v = CUDART_NAN;
                a.features_out[traj * a.n_features + c] = v;
            }
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

__device__ __forceinline__ int64_t traj_at(const pb_solve_args& a, int64_t q)
{
    return a.order ? static_cast<int64_t>(__ldg(a.order + q)) : q;
}

template <class Sys>
__device__ __forceinline__ Stats<Sys::S> stats_slot(unsigned char* smem, bool with_stats)
{
    Stats<Sys::S> st;
    if (!with_stats) {
        st.d = nullptr;
        st.i = nullptr;
        st.nthr = 0;
        st.tid = 0;
        return st;
    }
    st.nthr = blockDim.x;
    st.tid = threadIdx.x;
    st.d = reinterpret_cast<double*>(smem);
    st.i = reinterpret_cast<int*>(smem + static_cast<size_t>(6 * Sys::S * 8) * blockDim.x);
    return st;
}

// Plain schedule: one thread per trajectory, no queue (the FP64 baseline when
// R = double).  DEFER selects the first pass of the deferred dense output.
template <class Sys, class R, bool DEFER>
__global__ void __launch_bounds__(256) k_solve_plain(const pb_solve_args a)
{
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ Plan pl;
    if (threadIdx.x == 0) build_plan(pl, a);
    __syncthreads();
    using I = Integrator<Sys, R>;
    const int64_t q = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q >= a.n_traj) return;
    const int64_t traj = traj_at(a, q);
    if (traj < 0 || traj >= a.n_traj) return;  // an order entry out of range is ignored
    auto st = stats_slot<Sys>(smem, !DEFER);
    typename I::L_t L;
    I::begin(L, st, traj, a);
    while (!I::template step<DEFER>(L, st, pl, traj, a)) {
    }
    I::template finish<DEFER>(L, st, pl, traj, a);
}

// Queue schedule: persistent warps take 32 consecutive queue positions at a time
// (one atomicAdd per warp) and come back for the next 32 once all their lanes
// are done.  Taking whole warps keeps the lanes of a warp on neighbouring
// positions of the processing order (spatially coherent ICs), which a per-lane
// refill would scatter.  With `redo_only`, only trajectories whose deferred
// records overflowed are integrated (inline).  Every loop is bounded: each
// trajectory runs at most max_steps attempted steps and the queue holds n_traj
// entries.
//
// PHASE (deferred dense output only): 0 = whole span; 1 = probe phase, which
// stops each trajectory at the first accepted or rejected step ending at or after
// t0 + kProbeFraction (t1 - t0), saves its state and writes its step count as a
// sort key; 2 = main phase, which takes trajectories in the sorted order and
// resumes them.  The probe does not clip the step at its end, so the sequence of
// steps, and every output, is the one of PHASE 0.
constexpr double kProbeFraction = 0.05;

// Main phase without sampling: the window is sampled by the next launch.
struct NoDrain {
    static constexpr bool kOn = false;
    __device__ static void publish(const pb_solve_args&, const Plan&, int64_t) {}
    __device__ static void drain(const pb_solve_args&, const Plan&, int) {}
};

// Drain (PHASE 2): each finished trajectory is published (Drain::publish, per
// lane); a warp that finds the queue empty samples published trajectories
// (Drain::drain) while the longest ones are still integrating.
template <class Sys, class R, bool DEFER, int PHASE = 0, class Drain = NoDrain>
__global__ void __launch_bounds__(256) k_solve_queue(const pb_solve_args a, int redo_only)
{
    static_assert(PHASE == 0 || DEFER, "the probed schedule saves no inline statistics");
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ Plan pl;
    if (threadIdx.x == 0) build_plan(pl, a);
    __syncthreads();
    using I = Integrator<Sys, R>;
    const int lane = threadIdx.x & 31;
    auto st = stats_slot<Sys>(smem, !DEFER);
    const double t_probe = a.t0 + kProbeFraction * (a.t1 - a.t0);
    // Refill threshold (work-queue compaction): with refill_lanes r in [1, 32), a warp
    // fetches new queue positions for its idle lanes as soon as r of them are idle,
    // so lanes whose trajectories finished early or stopped (diverged, unbounded)
    // take new work while their neighbours keep integrating.  The lanes fetched
    // together take consecutive positions of the processing order.  r = 32 (or 0) is
    // the whole-warp schedule below; the probe phase always uses it.
    const int refill = (a.refill_lanes > 0 && a.refill_lanes < 32) ? a.refill_lanes : 32;
    if (PHASE != 1 && refill < 32) {
        typename I::L_t L;
        int64_t traj = -1;
        bool active = false, exhausted = false;
        while (true) {
            const unsigned idle = __ballot_sync(0xffffffffu, !active);
            if (!exhausted && __popc(idle) >= refill) {
                const int leader = __ffs(idle) - 1;
                unsigned long long base = 0;
                if (lane == leader) base = atomicAdd(a.queue_counter, static_cast<unsigned long long>(__popc(idle)));
                base = __shfl_sync(0xffffffffu, base, leader);
                if (static_cast<int64_t>(base) >= a.n_traj) exhausted = true;
                const int64_t q = static_cast<int64_t>(base) + __popc(idle & ((1u << lane) - 1u));
                if (!active && q < a.n_traj) {
                    traj = PHASE == 2 ? static_cast<int64_t>(sort_vec(a, pl.sl.val_out_off)[q]) : traj_at(a, q);
                    const bool in_range = traj >= 0 && traj < a.n_traj;  // an order entry out of range is ignored
                    const bool skip = !in_range ||
                                      (redo_only && reinterpret_cast<const int*>(tail_ptr(a, pl.sl, traj))[0] >= 0);
                    if (!skip) {
                        if (PHASE == 2) {
                            active = I::resume(L, pl, traj, a);
                        } else {
                            I::begin(L, st, traj, a);
                            active = true;
                        }
                    }
                    if constexpr (PHASE == 2 && Drain::kOn)
                        if (!active) Drain::publish(a, pl, skip ? -1 : traj);  // skipped, or done in the probe
                }
            }
            if (exhausted && __ballot_sync(0xffffffffu, active) == 0u) break;
            if (active && I::template step<DEFER>(L, st, pl, traj, a)) {
                I::template finish<DEFER>(L, st, pl, traj, a);
                if constexpr (PHASE == 2 && Drain::kOn) Drain::publish(a, pl, traj);
                active = false;
            }
        }
        if constexpr (Drain::kOn) Drain::drain(a, pl, lane);
        return;
    }
    while (true) {
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(a.queue_counter, 32ull);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (static_cast<int64_t>(base) >= a.n_traj) {
            if constexpr (Drain::kOn) Drain::drain(a, pl, lane);
            break;
        }
        const int64_t q = static_cast<int64_t>(base) + lane;
        if (q < a.n_traj) {
            const int64_t traj = PHASE == 2 ? static_cast<int64_t>(sort_vec(a, pl.sl.val_out_off)[q]) : traj_at(a, q);
            const bool in_range = traj >= 0 && traj < a.n_traj;  // an order entry out of range is ignored
            const bool skip = !in_range ||
                              (redo_only && reinterpret_cast<const int*>(tail_ptr(a, pl.sl, traj))[0] >= 0);
            unsigned key = 0;
            if (!skip) {
                typename I::L_t L;
                if (PHASE == 2) {
                    if (I::resume(L, pl, traj, a)) {
                        while (!I::template step<DEFER>(L, st, pl, traj, a)) {
                        }
                        I::template finish<DEFER>(L, st, pl, traj, a);
                    }
                    if constexpr (Drain::kOn) Drain::publish(a, pl, traj);
                } else if (PHASE == 1) {
                    I::begin(L, st, traj, a);
                    bool done = false;
                    while (!done && L.t < t_probe) done = I::template step<DEFER>(L, st, pl, traj, a);
                    if (done) I::template finish<DEFER>(L, st, pl, traj, a);
                    I::save(L, pl, traj, a, done ? 1 : 0);
                    key = done ? 0u : static_cast<unsigned>(L.steps);
                } else {
                    I::begin(L, st, traj, a);
                    while (!I::template step<DEFER>(L, st, pl, traj, a)) {
                    }
                    I::template finish<DEFER>(L, st, pl, traj, a);
                }
            }
            if constexpr (PHASE == 2 && Drain::kOn)
                if (skip) Drain::publish(a, pl, -1);
            if (PHASE == 1) {
                sort_vec(a, pl.sl.key_in_off)[q] = key;
                sort_vec(a, pl.sl.val_in_off)[q] = static_cast<unsigned>(traj);
            }
        }
        __syncwarp();
    }
}

}  // namespace pb
