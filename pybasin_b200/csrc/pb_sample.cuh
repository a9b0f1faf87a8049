// Second pass of the deferred dense output: evaluate every save point of the
// feature window from the step records and reduce the window statistics.
//
// One warp per trajectory; lane l evaluates save points win_begin + l,
// win_begin + l + 32, ...  Each lane walks the (time-ordered) records of its
// trajectory forward to the record that covers its save point, so all 32 lanes
// stay busy on the same trajectory regardless of how many save points a step
// covers.  The statistics match the inline path (torch_features_statistical.py
// :30-110,:307-318 and torch_features_pattern.py:56-60 of the reference): a
// shifted sum and sum of squares (shift = first window sample), min, max, last
// sample, NaN flags and level crossings between consecutive samples, reduced
// across the warp with shuffles.
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
        default: return CUDART_NAN;
    }
}

template <class R, int S>
__global__ void __launch_bounds__(256) k_sample(const pb_solve_args a)
{
    __shared__ Plan pl;
    if (threadIdx.x == 0) build_plan(pl, a);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t traj = static_cast<int64_t>(blockIdx.x) * (blockDim.x >> 5) + warp;
    if (traj >= a.n_traj) return;  // warp-uniform
    const unsigned char* tl = tail_ptr(a, pl.sl, traj);
    const int nrec = reinterpret_cast<const int*>(tl)[0];
    if (nrec < 0) return;  // integrated again by the inline pass
    const double* fill = reinterpret_cast<const double*>(tl + 16);
    const int ns = pl.ns;
    const int64_t nwin = a.n_save - a.win_begin;

    double sh[S], s1[S], s2[S], mn[S], mx[S], last[S];
#pragma unroll
    for (int k = 0; k < S; ++k) {
        sh[k] = 0.0;
        s1[k] = 0.0;
        s2[k] = 0.0;
        mn[k] = CUDART_INF;
        mx[k] = -CUDART_INF;
        last[k] = 0.0;
    }
    int nan_flags = 0;
    int cross_cnt[PB_MAX_CROSSING] = {0, 0, 0, 0};
    double carry[PB_MAX_CROSSING] = {0.0, 0.0, 0.0, 0.0};  // previous sample of each crossing state

    int k = 0;           // record under this lane's save point
    int loaded = -1;     // record whose data sits in registers
    int rsi = 0, rns = 0;
    double rt = 0.0, rdt = 1.0;
    R co[5 * S];
    if (nrec > 0) {
        const int* hi = reinterpret_cast<const int*>(record_ptr(a, pl.sl, traj, 0) + 16);
        rsi = hi[0];
        rns = hi[1];
    }
    for (int64_t base = a.win_begin; base < a.n_save; base += 32) {
        const int j = static_cast<int>(base) + lane;
        const bool valid = j < a.n_save;
        double v[S];
#pragma unroll
        for (int q = 0; q < S; ++q) v[q] = 0.0;
        if (valid) {
            while (k < nrec && j >= rsi + rns) {
                ++k;
                if (k < nrec) {
                    const int* hi = reinterpret_cast<const int*>(record_ptr(a, pl.sl, traj, k) + 16);
                    rsi = hi[0];
                    rns = hi[1];
                }
            }
            if (k < nrec && j >= rsi) {
                if (loaded != k) {
                    const unsigned char* rec = record_ptr(a, pl.sl, traj, k);
                    rt = reinterpret_cast<const double*>(rec)[0];
                    rdt = reinterpret_cast<const double*>(rec)[1];
                    const R* c = reinterpret_cast<const R*>(rec + kRecordHeader);
#pragma unroll
                    for (int q = 0; q < 5 * S; ++q) {
                        co[q] = R(0);
                        if (q < 5 * ns) co[q] = c[q];
                    }
                    loaded = k;
                }
                const double ts = __ldg(a.save_ts + j);
                const R x = (ts <= rt + dp::save_slack) ? R(0) : static_cast<R>((ts - rt) / rdt);
#pragma unroll
                for (int q = 0; q < S; ++q) {
                    const R y = co[5 * q], hk = co[5 * q + 1], cc = co[5 * q + 2], bb = co[5 * q + 3],
                            aa = co[5 * q + 4];
                    v[q] = static_cast<double>(y + x * (hk + x * (cc + x * (bb + x * aa))));
                }
            } else {
#pragma unroll
                for (int q = 0; q < S; ++q)
                    if (q < ns) v[q] = fill[pl.stat_state[q]];
            }
        }
        if (base == a.win_begin) {  // shift = first window sample (lane 0 holds it)
#pragma unroll
            for (int q = 0; q < S; ++q) {
                const double f = __shfl_sync(0xffffffffu, v[q], 0);
                sh[q] = isfinite(f) ? f : 0.0;
            }
        }
        if (valid) {
#pragma unroll
            for (int q = 0; q < S; ++q) {
                if (q >= ns) continue;
                const double d = v[q] - sh[q];
                s1[q] += d;
                s2[q] = fma(d, d, s2[q]);
                mn[q] = fmin(mn[q], v[q]);
                mx[q] = fmax(mx[q], v[q]);
                if (v[q] != v[q]) nan_flags |= 1 << q;
                if (j == a.n_save - 1) last[q] = v[q];
            }
            for (int m = 0; m < pl.n_med; ++m)
                median_ptr(a, pl.sl)[(traj * pl.n_med + m) * nwin + (j - a.win_begin)] =
                    static_cast<float>(pick(v, pl.slot_of[pl.med_state[m]]));
        }
        for (int c = 0; c < pl.n_cross; ++c) {
            const double cur = pick(v, pl.slot_of[pl.cross_state[c]]);
            double prev = __shfl_up_sync(0xffffffffu, cur, 1);
            if (lane == 0) prev = carry[c];
            const bool count_it = valid && j > a.win_begin;
            const bool changed = (cur > pl.cross_level[c]) != (prev > pl.cross_level[c]);
            const int inc = (count_it && changed) ? 1 : 0;
#pragma unroll
            for (int q = 0; q < PB_MAX_CROSSING; ++q) cross_cnt[q] += (q == c) ? inc : 0;
            const double nxt = __shfl_sync(0xffffffffu, cur, 31);
#pragma unroll
            for (int q = 0; q < PB_MAX_CROSSING; ++q) carry[q] = (q == c) ? nxt : carry[q];
        }
    }
    // warp reductions
#pragma unroll
    for (int q = 0; q < S; ++q) {
        for (int o = 16; o > 0; o >>= 1) {
            s1[q] += __shfl_xor_sync(0xffffffffu, s1[q], o);
            s2[q] += __shfl_xor_sync(0xffffffffu, s2[q], o);
            mn[q] = fmin(mn[q], __shfl_xor_sync(0xffffffffu, mn[q], o));
            mx[q] = fmax(mx[q], __shfl_xor_sync(0xffffffffu, mx[q], o));
            last[q] += __shfl_xor_sync(0xffffffffu, last[q], o);  // one lane holds it, the rest 0
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        nan_flags |= __shfl_xor_sync(0xffffffffu, nan_flags, o);
#pragma unroll
        for (int q = 0; q < PB_MAX_CROSSING; ++q) cross_cnt[q] += __shfl_xor_sync(0xffffffffu, cross_cnt[q], o);
    }
    if (lane != 0 || !a.features_out) return;
    const double n = static_cast<double>(nwin);
    int jc = 0;
    for (int c = 0; c < a.n_features; ++c) {
        const int kind = a.feat_kind[c];
        if (kind == PB_FEAT_MEDIAN) continue;  // written by the median pass
        const int slot = pl.slot_of[a.feat_state[c]];
        const bool has_nan = (nan_flags >> slot) & 1;
        double cr = CUDART_NAN;
        if (kind == PB_FEAT_CROSSINGS) {
            cr = jc < pl.n_cross ? static_cast<double>(pick(cross_cnt, jc)) : CUDART_NAN;
            ++jc;
        }
        double v = feature_value(kind, pick(sh, slot), pick(s1, slot), pick(s2, slot),
                                 has_nan ? CUDART_NAN : pick(mn, slot), has_nan ? CUDART_NAN : pick(mx, slot),
                                 pick(last, slot), n, cr);
        if (nwin <= 0) v = CUDART_NAN;
        a.features_out[traj * a.n_features + c] = v;
    }
}

}  // namespace pb
