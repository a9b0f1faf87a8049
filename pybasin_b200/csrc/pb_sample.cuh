// Second pass of the deferred dense output: evaluate every save point of the
// feature window from the step records and reduce the window statistics.
//
// One warp per trajectory; lane l takes records l, l + 32, ... of its
// trajectory and evaluates the save points each record's step covers (no search,
// no shuffles inside the sample loop).  The statistics match the inline path
// (torch_features_statistical.py:30-110,307-318 and torch_features_pattern.py
// :56-60 of the reference): a shifted sum and sum of squares (shift = first
// window sample), min, max, last sample, NaN flags and level crossings between
// consecutive samples, reduced across the warp with shuffles.
//
// The kernels are templated on the number of feature states NS (not on the
// system), so every system, built-in or compiled at run time, shares them.  In
// the FP32 pass the offset of a save point from its step start, ts - t, comes
// from a (hi, lo) float split of both times (exact to a few float ulps of the
// offset), so the sample loop runs without FP64 arithmetic or conversions.
#pragma once
#include "pb_dopri5.cuh"

namespace pb {

__device__ __forceinline__ double feature_value(int kind, double sh, double s1, double s2, double mn, double mx,
                                                double last, double n, double crossings)
{
    const double mean = sh + s1 / n;
    const double var = fmax((s2 - s1 * (s1 / n)) / n, 0.0);
    switch (kind) {
        case PB_FEAT_MEAN: return mean;
        case PB_FEAT_STD: return sqrt(var);
        case PB_FEAT_VAR: return var;
        case PB_FEAT_RMS: return sqrt((s2 + sh * (2.0 * s1 + n * sh)) / n);
        case PB_FEAT_MAX: return mx;
        case PB_FEAT_ABSMAX: return fmax(fabs(mx), fabs(mn));
        case PB_FEAT_MIN: return mn;
        case PB_FEAT_DELTA: return fabs(mx - mean);
        case PB_FEAT_LOG_DELTA: return log(fabs(mx - mean) + 1e-10);
        case PB_FEAT_AMPLITUDE: return mx - mn;
        case PB_FEAT_CROSSINGS: return crossings;
        case PB_FEAT_LAST: return last;
        case PB_FEAT_SUM: return n * sh + s1;
        case PB_FEAT_ABS_ENERGY: return s2 + sh * (2.0 * s1 + n * sh);
        case PB_FEAT_LENGTH: return n;
        case PB_FEAT_VARIATION_COEFF: return sqrt(var) / (fabs(mean) + 1e-10);
        default: return CUDART_NAN;
    }
}

// y(t + x dt) from a record's coefficients [y, h*k1, c, b, a] (Horner form)
template <class R>
__device__ __forceinline__ R dense_value(const R* c, R x)
{
    return fmad(x, fmad(x, fmad(x, fmad(x, c[4], c[3]), c[2]), c[1]), c[0]);
}

// Per-lane window statistics accumulated by the sampling pass.
template <int NS>
struct SampleAcc {
    double sh[NS], s1[NS], s2[NS], mn[NS], mx[NS], last[NS];
    int nan_flags;
    int cross_cnt[PB_MAX_CROSSING];
    double carry[PB_MAX_CROSSING];  // previous sample of each crossing state (the one before lane 0's)
    bool shift_set;
};

// Fold one batch of (up to 32) consecutive save points into the accumulators
// (the fill values after a stop).  Lane l holds sample j = j0 + l (valid if
// l < nvalid).  Collective over the warp.
template <int NS>
__device__ __forceinline__ void fold_samples(SampleAcc<NS>& acc, const Plan& pl, const pb_solve_args& a,
                                             int64_t traj, int64_t nwin, int j0, int nvalid, const double (&v)[NS],
                                             int lane)
{
    const int j = j0 + lane;
    const bool valid = lane < nvalid;
    if (!acc.shift_set) {  // shift = first window sample (lane 0 of the first batch)
#pragma unroll
        for (int q = 0; q < NS; ++q) {
            const double f = __shfl_sync(0xffffffffu, v[q], 0);
            acc.sh[q] = isfinite(f) ? f : 0.0;
        }
        acc.shift_set = true;
    }
    if (valid) {
#pragma unroll
        for (int q = 0; q < NS; ++q) {
            const double d = v[q] - acc.sh[q];
            acc.s1[q] += d;
            acc.s2[q] = fma(d, d, acc.s2[q]);
            acc.mn[q] = fmin(acc.mn[q], v[q]);
            acc.mx[q] = fmax(acc.mx[q], v[q]);
            if (v[q] != v[q]) acc.nan_flags |= 1 << q;
            if (j == a.n_save - 1) acc.last[q] = v[q];
        }
        for (int m = 0; m < pl.n_med; ++m)
            median_ptr(a, pl.sl)[(traj * pl.n_med + m) * nwin + (j - a.win_begin)] =
                static_cast<float>(pick(v, pl.slot_of[pl.med_state[m]]));
    }
    const int lastl = nvalid - 1;
    for (int c = 0; c < pl.n_cross; ++c) {
        const double cur = pick(v, pl.slot_of[pl.cross_state[c]]);
        double prev = __shfl_up_sync(0xffffffffu, cur, 1);
        if (lane == 0) prev = pick(acc.carry, c);
        const bool changed = (cur > pl.cross_level[c]) != (prev > pl.cross_level[c]);
        const int inc = (valid && j > a.win_begin && changed) ? 1 : 0;
        const double nxt = __shfl_sync(0xffffffffu, cur, lastl);
#pragma unroll
        for (int q = 0; q < PB_MAX_CROSSING; ++q) {
            acc.cross_cnt[q] += (q == c) ? inc : 0;
            acc.carry[q] = (q == c) ? nxt : acc.carry[q];
        }
    }
}

// (hi, lo) float split of the save grid, for the FP32 sampling pass
__global__ void __launch_bounds__(256) k_split_saves(const double* __restrict__ ts, int n, float2* __restrict__ out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double t = ts[i];
    const float hi = static_cast<float>(t);
    out[i] = make_float2(hi, static_cast<float>(t - static_cast<double>(hi)));
}

// Step-local offset x = (ts - t) / dt of save point j in a record starting at t.
// FP32: from the split grid and the split record start; FP64: directly.
struct OffsetF32 {
    const float2* grid;
    float t_hi, t_lo, inv_dt;
    __device__ __forceinline__ OffsetF32(const float2* g, double t, double idt) : grid(g)
    {
        t_hi = static_cast<float>(t);
        t_lo = static_cast<float>(t - static_cast<double>(t_hi));
        inv_dt = static_cast<float>(idt);
    }
    __device__ __forceinline__ float at(int j) const
    {
        const float2 s = grid[j];
        const float d = (s.x - t_hi) + (s.y - t_lo);
        return d <= 1e-12f ? 0.f : d * inv_dt;  // save slack of dopri5_generic.zig:197
    }
};
struct OffsetF64 {
    const double* grid;
    double t, inv_dt;
    __device__ __forceinline__ OffsetF64(const double* g, double t0, double idt) : grid(g), t(t0), inv_dt(idt) {}
    __device__ __forceinline__ double at(int j) const
    {
        const double ts = __ldg(grid + j);
        return ts <= t + dp::save_slack ? 0.0 : (ts - t) * inv_dt;
    }
};

template <class R>
struct OffsetOf {
    using type = OffsetF64;
    __device__ __forceinline__ static OffsetF64 make(const float2*, const double* ts, double t, double idt)
    {
        return OffsetF64(ts, t, idt);
    }
};
template <>
struct OffsetOf<float> {
    using type = OffsetF32;
    __device__ __forceinline__ static OffsetF32 make(const float2* split, const double*, double t, double idt)
    {
        return OffsetF32(split, t, idt);
    }
};

// NC = crossing states compiled in (0 when no column counts crossings, which
// keeps the per-lane crossing registers out of the common case).
// Sampling of one trajectory by the calling warp (all 32 lanes, warp-uniform traj).
// What the integrator wrote (tail, records) is read through L2 (__ldcg): when the
// sampling is drained into the main phase, another SM wrote it during this launch.
template <class R, int NS, int NC>
__device__ __forceinline__ void sample_trajectory(const pb_solve_args& a, const Plan& pl, int64_t traj, int lane)
{
    const unsigned char* tl = tail_ptr(a, pl.sl, traj);
    const int nrec = __ldcg(reinterpret_cast<const int*>(tl));
    if (nrec < 0) return;  // integrated again by the inline pass
    const int si_end = __ldcg(reinterpret_cast<const int*>(tl) + 1);
    const double* fill = reinterpret_cast<const double*>(tl + 16);
    const int64_t nwin = a.n_save - a.win_begin;
    const float2* split = reinterpret_cast<const float2*>(static_cast<const unsigned char*>(a.scratch) + pl.sl.split_off);

    SampleAcc<NS> acc;
#pragma unroll
    for (int q = 0; q < NS; ++q) {
        acc.sh[q] = 0.0;
        acc.s1[q] = 0.0;
        acc.s2[q] = 0.0;
        acc.mn[q] = CUDART_INF;
        acc.mx[q] = -CUDART_INF;
        acc.last[q] = 0.0;
    }
    acc.nan_flags = 0;
#pragma unroll
    for (int q = 0; q < PB_MAX_CROSSING; ++q) {
        acc.cross_cnt[q] = 0;
        acc.carry[q] = 0.0;
    }
    acc.shift_set = false;

    // records, 32 at a time: lane i takes record chunk+i (coalesced loads of
    // consecutive records) and evaluates the save points its step covers, in
    // time order.  Every record covers at least one save point.  Per-record
    // partial sums are kept in R and folded into the lane's FP64 sums once per
    // record; crossings between the last sample of one lane and the first of the
    // next are counted after the loop with one shuffle per crossing state.
    for (int chunk = 0; chunk < nrec; chunk += 32) {
        const int k = chunk + lane;
        const int hl = min(31, nrec - 1 - chunk);  // last lane holding a record
        const bool have = k < nrec;
        double rt = 0.0, rdt = 0.0;
        R co[5 * NS];
        int rsi = 0, rn = 0;
#pragma unroll
        for (int q = 0; q < 5 * NS; ++q) co[q] = R(0);
        if (have) {
            const unsigned char* rec = record_ptr(a, pl.sl, traj, k);
            rt = __ldcg(reinterpret_cast<const double*>(rec));
            rdt = 1.0 / __ldcg(reinterpret_cast<const double*>(rec) + 1);
            const int2 span = __ldcg(reinterpret_cast<const int2*>(rec + kRecordIndexOffset));
            rsi = span.x;
            rn = span.y;
            const R* c = reinterpret_cast<const R*>(rec + kRecordHeader);
#pragma unroll
            for (int q = 0; q < 5 * NS; ++q) co[q] = __ldcg(c + q);
        }
        const auto off = OffsetOf<R>::make(split, a.save_ts, rt, rdt);
        if (!acc.shift_set) {  // shift = first window sample = first save of record 0 (lane 0)
            const R x = static_cast<R>(off.at(rsi));
#pragma unroll
            for (int q = 0; q < NS; ++q) {
                const double f = __shfl_sync(0xffffffffu, static_cast<double>(dense_value(co + 5 * q, x)), 0);
                acc.sh[q] = isfinite(f) ? f : 0.0;
            }
            acc.shift_set = true;
        }
        R p1[NS], p2[NS], pmn[NS], pmx[NS], sh[NS], vlast[NS];
#pragma unroll
        for (int q = 0; q < NS; ++q) {
            p1[q] = R(0);
            p2[q] = R(0);
            pmn[q] = R(CUDART_INF);
            pmx[q] = R(-CUDART_INF);
            sh[q] = static_cast<R>(acc.sh[q]);
            vlast[q] = R(0);
        }
        double cfirst[NC > 0 ? NC : 1], cprev[NC > 0 ? NC : 1];
        int ccnt[NC > 0 ? NC : 1];
#pragma unroll
        for (int c = 0; c < (NC > 0 ? NC : 1); ++c) {
            cfirst[c] = 0.0;
            cprev[c] = 0.0;
            ccnt[c] = 0;
        }
        const bool with_median = pl.n_med > 0;
        for (int i = 0; i < rn; ++i) {
            const int j = rsi + i;
            const R x = static_cast<R>(off.at(j));
            R v[NS];
#pragma unroll
            for (int q = 0; q < NS; ++q) {
                v[q] = dense_value(co + 5 * q, x);
                const R d = v[q] - sh[q];
                p1[q] += d;
                p2[q] = fmad(d, d, p2[q]);  // NaN here iff a sample is NaN (the shift is finite)
                pmn[q] = fmin(pmn[q], v[q]);
                pmx[q] = fmax(pmx[q], v[q]);
                vlast[q] = v[q];
            }
            if (with_median)
                for (int m = 0; m < pl.n_med; ++m)
                    median_ptr(a, pl.sl)[(traj * pl.n_med + m) * nwin + (j - a.win_begin)] =
                        static_cast<float>(pick(v, pl.slot_of[pl.med_state[m]]));
#pragma unroll
            for (int c = 0; c < NC; ++c) {
                if (c >= pl.n_cross) break;
                const double cur = static_cast<double>(pick(v, pl.slot_of[pl.cross_state[c]]));
                const bool changed = (cur > pl.cross_level[c]) != (cprev[c] > pl.cross_level[c]);
                ccnt[c] += (i > 0 && changed) ? 1 : 0;
                cfirst[c] = (i == 0) ? cur : cfirst[c];
                cprev[c] = cur;
            }
        }
        const bool holds_last = have && rsi + rn == a.n_save;
#pragma unroll
        for (int q = 0; q < NS; ++q) {
            acc.s1[q] += static_cast<double>(p1[q]);
            acc.s2[q] += static_cast<double>(p2[q]);
            acc.mn[q] = fmin(acc.mn[q], static_cast<double>(pmn[q]));
            acc.mx[q] = fmax(acc.mx[q], static_cast<double>(pmx[q]));
            if (p2[q] != p2[q]) acc.nan_flags |= 1 << q;
            if (holds_last) acc.last[q] = static_cast<double>(vlast[q]);
        }
        // crossings across record boundaries: lane l's first sample against lane
        // l-1's last (lane 0 against the carry from the previous chunk)
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            if (c >= pl.n_cross) break;
            double prev = __shfl_up_sync(0xffffffffu, cprev[c], 1);
            if (lane == 0) prev = acc.carry[c];
            const bool changed = (cfirst[c] > pl.cross_level[c]) != (prev > pl.cross_level[c]);
            acc.cross_cnt[c] += ccnt[c] + ((have && rsi > a.win_begin && changed) ? 1 : 0);
            acc.carry[c] = __shfl_sync(0xffffffffu, cprev[c], hl);
        }
    }
    // save points after the last record: the trajectory stopped (or t1 was reached
    // before them); they hold the fill value (+inf after an unbounded stop)
    const int tail0 = max(si_end, static_cast<int>(a.win_begin));
    for (int j0 = tail0; j0 < a.n_save; j0 += 32) {
        const int nvalid = min(32, a.n_save - j0);
        double v[NS];
#pragma unroll
        for (int q = 0; q < NS; ++q) v[q] = __ldcg(fill + pl.stat_state[q]);
        fold_samples(acc, pl, a, traj, nwin, j0, nvalid, v, lane);
    }
    // warp reductions
#pragma unroll
    for (int q = 0; q < NS; ++q) {
        for (int o = 16; o > 0; o >>= 1) {
            acc.s1[q] += __shfl_xor_sync(0xffffffffu, acc.s1[q], o);
            acc.s2[q] += __shfl_xor_sync(0xffffffffu, acc.s2[q], o);
            acc.mn[q] = fmin(acc.mn[q], __shfl_xor_sync(0xffffffffu, acc.mn[q], o));
            acc.mx[q] = fmax(acc.mx[q], __shfl_xor_sync(0xffffffffu, acc.mx[q], o));
            acc.last[q] += __shfl_xor_sync(0xffffffffu, acc.last[q], o);  // one lane holds it, the rest 0
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        acc.nan_flags |= __shfl_xor_sync(0xffffffffu, acc.nan_flags, o);
#pragma unroll
        for (int q = 0; q < PB_MAX_CROSSING; ++q)
            acc.cross_cnt[q] += __shfl_xor_sync(0xffffffffu, acc.cross_cnt[q], o);
    }
    if (lane != 0 || !a.features_out) return;
    const double n = static_cast<double>(nwin);
    int jc = 0;
    for (int c = 0; c < a.n_features; ++c) {
        const int kind = a.feat_kind[c];
        if (PB_FEAT_IS_WINDOW(kind)) continue;  // written by the window pass
        const int slot = pl.slot_of[a.feat_state[c]];
        const bool has_nan = (acc.nan_flags >> slot) & 1;
        double cr = CUDART_NAN;
        if (kind == PB_FEAT_CROSSINGS) {
            cr = jc < pl.n_cross ? static_cast<double>(pick(acc.cross_cnt, jc)) : CUDART_NAN;
            ++jc;
        }
        const double v = feature_value(kind, pick(acc.sh, slot), pick(acc.s1, slot), pick(acc.s2, slot),
                                       has_nan ? CUDART_NAN : pick(acc.mn, slot),
                                       has_nan ? CUDART_NAN : pick(acc.mx, slot), pick(acc.last, slot), n, cr);
        a.features_out[traj * a.n_features + c] = v;
    }
}

template <class R, int NS, int NC>
__global__ void __launch_bounds__(128) k_sample(const pb_solve_args a)
{
    __shared__ Plan pl;
    if (threadIdx.x == 0) build_plan(pl, a);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t traj = static_cast<int64_t>(blockIdx.x) * (blockDim.x >> 5) + warp;
    if (traj >= a.n_traj || pl.ns != NS) return;  // warp-uniform
    if (pl.sl.probed && drain_sampled(a, pl.sl, a.n_traj)[traj]) return;  // sampled by the main phase
    sample_trajectory<R, NS, NC>(a, pl, traj, lane);
}

// Sampling drained into the probed main phase (k_solve_queue's Drain).  A lane
// that finishes a trajectory publishes it: after a fence (its records and tail
// are visible device-wide), it takes the next slot of the published list and
// stores the id + 1 there (a skipped queue position stores -1).  A
// warp that finds the queue empty claims slots in order and samples each one's
// trajectory once it is published, while the longest trajectories still
// integrate.  Every wait is bounded: a warp that waits longer than kMaxPolls
// polls for a slot stops draining, and the sampling pass after the launch takes
// every trajectory whose sampled flag is not set.  Producers never wait, so no
// lane depends on a waiting warp.
constexpr int kMaxPolls = 1 << 17;

template <class R, int NS>
struct SampleDrain {
    static constexpr bool kOn = true;
    __device__ static void publish(const pb_solve_args& a, const Plan& pl, int64_t traj)
    {
        __threadfence();
        unsigned long long* cnt = drain_counters(a, pl.sl);
        const unsigned long long slot = atomicAdd(cnt, 1ull);
        if (slot < static_cast<unsigned long long>(a.n_traj))
            atomicExch(drain_list(a, pl.sl) + slot, traj >= 0 ? static_cast<int>(traj) + 1 : -1);
    }
    __device__ static void drain(const pb_solve_args& a, const Plan& pl, int lane)
    {
        if (pl.ns != NS || pl.n_cross > 0) return;  // warp-uniform: the sampling pass covers it
        unsigned long long* cnt = drain_counters(a, pl.sl);
        int* list = drain_list(a, pl.sl);
        unsigned char* sampled = drain_sampled(a, pl.sl, a.n_traj);
        while (true) {
            unsigned long long slot = 0;
            if (lane == 0) slot = atomicAdd(cnt + 1, 1ull);
            slot = __shfl_sync(0xffffffffu, slot, 0);
            if (slot >= static_cast<unsigned long long>(a.n_traj)) return;
            int v = 0;
            if (lane == 0) {
                for (int poll = 0; poll < kMaxPolls; ++poll) {
                    v = atomicAdd(list + slot, 0);
                    if (v != 0) break;
                    __nanosleep(256);
                }
            }
            v = __shfl_sync(0xffffffffu, v, 0);
            if (v == 0) return;  // gave up: the sampling pass takes what is left
            __threadfence();
            if (v > 0) {
                sample_trajectory<R, NS, 0>(a, pl, v - 1, lane);
                __syncwarp();
                if (lane == 0) sampled[v - 1] = 1;
            }
        }
    }
};

}  // namespace pb
