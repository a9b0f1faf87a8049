// C ABI of the B200 fused Dopri5 + feature library: argument checks, kernel
// selection (system x precision x schedule), the median pass and 1-NN labelling.
#include <cuda_runtime.h>
#include <math_constants.h>
#include <stdint.h>

#include <cub/device/device_radix_sort.cuh>

#include "pb_network.cuh"
#include "pb_sample.cuh"
#include "pb_launch.h"
#include "pybasin_b200.h"

namespace pb {

// ---------------------------------------------------------------------------
// exact lower median of a window row (torch.median semantics: the lower of the
// two middle values, NaN if the row holds a NaN), by 4-pass radix select on
// order-preserving 32-bit keys.  One warp per (trajectory, median column).
// ---------------------------------------------------------------------------
struct MedianPlan {
    int n_med;                       // window columns
    int col[PB_MAX_FEATURES];        // output column of window column m
    int kind[PB_MAX_FEATURES];       // its feature kind
    double param[PB_MAX_FEATURES];   // and parameter (q, t, n, lag, r)
    double param2[PB_MAX_FEATURES];  // second parameter of the two-parameter kinds
    int peak_idx[PB_MAX_FEATURES];   // NUMBER_PEAKS columns: index among them (orbit data), else -1
    int n_peak_cols;
    int peak_cap;
    double* peaks_out;               // (n_traj, n_peak_cols, peak_cap) or NULL
    int n_sorted;                    // window columns of the sorted kinds (PB_FEAT_IS_SORTED)
    int sorted_m[PB_MAX_FEATURES];   // their window column indices m
    int n_spectral;                  // window columns of the spectral kinds (PB_FEAT_IS_SPECTRAL)
    int spectral_m[PB_MAX_FEATURES];
    int n_symbolic;                  // window columns of the symbolic kinds (PB_FEAT_IS_SYMBOLIC)
    int symbolic_m[PB_MAX_FEATURES];
};

__device__ __forceinline__ uint32_t float_key(float f)
{
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float key_float(uint32_t k)
{
    const uint32_t u = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
    return __uint_as_float(u);
}

// k-th smallest (0-based) value of a NaN-free row, by a 4-pass 8-bit radix select
// on order-preserving keys (warp-collective; h = 256 bins of this warp)
__device__ float select_rank(const float* __restrict__ x, int nwin, unsigned k, unsigned* h, int lane)
{
    uint32_t prefix = 0, prefix_mask = 0;
    for (int pass = 0; pass < 4; ++pass) {
        const int shift = 24 - 8 * pass;
        for (int b = lane; b < 256; b += 32) h[b] = 0;
        __syncwarp();
        for (int i = lane; i < nwin; i += 32) {
            const uint32_t key = float_key(x[i]);
            if ((key & prefix_mask) == prefix) atomicAdd(&h[(key >> shift) & 0xffu], 1u);
        }
        __syncwarp();
        // lane 0 scans the 256 bins to find the bin holding rank k
        unsigned sel = 0, before = 0;
        if (lane == 0) {
            unsigned acc = 0;
            for (int b = 0; b < 256; ++b) {
                if (acc + h[b] > k) {
                    sel = static_cast<unsigned>(b);
                    before = acc;
                    break;
                }
                acc += h[b];
            }
        }
        sel = __shfl_sync(0xffffffffu, sel, 0);
        before = __shfl_sync(0xffffffffu, before, 0);
        k -= before;
        prefix |= sel << shift;
        prefix_mask |= 0xffu << shift;
        __syncwarp();
    }
    return key_float(prefix);
}

__device__ __forceinline__ double warp_sum_d(double v)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Least squares of a series a(0..cnt-1) on t = 0..cnt-1 (torch_features_trend.py:11-51),
// warp-collective: attr 0..4 = slope, intercept, rvalue, the reference's pseudo
// p-value 1 / (1 + |t|), stderr.  `a` is evaluated on demand (two or three passes).
template <class Series>
__device__ double warp_trend(const Series& a, int cnt, int attr, int lane)
{
    double s = 0.0;
    for (int i = lane; i < cnt; i += 32) s += a(i);
    const double am = warp_sum_d(s) / cnt, tm = 0.5 * (cnt - 1.0);
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
    for (int i = lane; i < cnt; i += 32) {
        const double dt = static_cast<double>(i) - tm, dx = a(i) - am;
        a0 += dt * dt;
        a1 += dt * dx;
        a2 += dx * dx;
    }
    const double ss_tt = warp_sum_d(a0), ss_tx = warp_sum_d(a1), ss_xx = warp_sum_d(a2);
    const double slope = ss_tx / (ss_tt + 1e-10), intercept = am - slope * tm;
    const double r = ss_tx / (sqrt(ss_tt * ss_xx) + 1e-10);
    if (attr == 0) return slope;
    if (attr == 1) return intercept;
    if (attr == 2) return r;
    if (attr == 3) return 1.0 / (1.0 + fabs(r * sqrt(cnt - 2.0) / (sqrt(1.0 - r * r) + 1e-10)));
    double rss = 0.0;
    for (int i = lane; i < cnt; i += 32) {
        const double e = a(i) - (slope * static_cast<double>(i) + intercept);
        rss += e * e;
    }
    return sqrt(warp_sum_d(rss) / (cnt - 2.0) / (ss_tt + 1e-10));
}

// Window pass: one warp per (trajectory, window column) computes the column's
// feature from the stored window (torch semantics of the reference calculators:
// median = lower middle value, quantile = linear interpolation, NaN in -> NaN out
// for order statistics, comparisons with NaN false).
__global__ void __launch_bounds__(256) k_window(const float* __restrict__ win, int64_t n_traj, int nwin,
                                                MedianPlan plan, double* __restrict__ out, int n_features)
{
    __shared__ __align__(16) unsigned hist[8][256];  // per warp: radix bins, or 128 doubles
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t row = static_cast<int64_t>(blockIdx.x) * 8 + warp;
    if (row >= n_traj * plan.n_med) return;  // warp-uniform
    const float* x = win + row * nwin;
    unsigned* h = hist[warp];
    const int64_t traj = row / plan.n_med;
    const int m = static_cast<int>(row - traj * plan.n_med);
    const int col = plan.col[m], kind = plan.kind[m];
    // warp-uniform; written by k_window_sorted / k_window_spectrum / k_window_symbolic
    if (PB_FEAT_IS_SORTED(kind) || PB_FEAT_IS_SPECTRAL(kind) || PB_FEAT_IS_SYMBOLIC(kind)) return;
    const double param = plan.param[m];
    const double n = static_cast<double>(nwin);
    double result = CUDART_NAN;
    if (kind == PB_FEAT_MEDIAN || kind == PB_FEAT_QUANTILE || kind == PB_FEAT_SYMMETRY_LOOKING) {
        bool nan_seen = false;
        for (int i = lane; i < nwin; i += 32) nan_seen |= isnan(x[i]);
        if (!__any_sync(0xffffffffu, nan_seen)) {
            if (kind == PB_FEAT_SYMMETRY_LOOKING) {  // |mean - median| < r * range, as 1 / 0
                double s = 0.0;
                float mx = -CUDART_INF_F, mn = CUDART_INF_F;
                for (int i = lane; i < nwin; i += 32) {
                    s += static_cast<double>(x[i]);
                    mx = fmaxf(mx, x[i]);
                    mn = fminf(mn, x[i]);
                }
                for (int off = 16; off > 0; off >>= 1) {
                    mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, off));
                    mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, off));
                }
                const double mean = warp_sum_d(s) / n;
                const double med = select_rank(x, nwin, static_cast<unsigned>((nwin - 1) / 2), h, lane);
                result = fabs(mean - med) < param * (static_cast<double>(mx) - static_cast<double>(mn)) ? 1.0 : 0.0;
            } else if (kind == PB_FEAT_MEDIAN) {
                result = select_rank(x, nwin, static_cast<unsigned>((nwin - 1) / 2), h, lane);
            } else {
                const double pos = param * (nwin - 1);
                const int lo = static_cast<int>(floor(pos));
                const int hi = lo + 1 < nwin ? lo + 1 : nwin - 1;
                const double va = select_rank(x, nwin, static_cast<unsigned>(lo), h, lane);
                const double vb = hi == lo ? va : select_rank(x, nwin, static_cast<unsigned>(hi), h, lane);
                result = va + (vb - va) * (pos - lo);
            }
        }
    } else {
        double s = 0.0;
        for (int i = lane; i < nwin; i += 32) s += static_cast<double>(x[i]);
        const double mean = warp_sum_d(s) / n;
        double a0 = 0.0, a1 = 0.0, a2 = 0.0;
        switch (kind) {
            case PB_FEAT_KURTOSIS:
            case PB_FEAT_SKEWNESS:
            case PB_FEAT_AUTOCORRELATION:
            case PB_FEAT_RATIO_BEYOND_R_SIGMA: {
                const int lag = static_cast<int>(param);
                for (int i = lane; i < nwin; i += 32) {
                    const double d = static_cast<double>(x[i]) - mean;
                    a0 += d * d;
                    if (kind == PB_FEAT_KURTOSIS || kind == PB_FEAT_SKEWNESS) {
                        a1 += d * d * d;
                        a2 += d * d * d * d;
                    } else if (kind == PB_FEAT_AUTOCORRELATION && lag > 0 && i + lag < nwin) {
                        a1 += d * (static_cast<double>(x[i + lag]) - mean);
                    }
                }
                const double m2 = warp_sum_d(a0);
                if (kind == PB_FEAT_KURTOSIS || kind == PB_FEAT_SKEWNESS) {
                    const double c2 = m2 / n, c3 = warp_sum_d(a1) / n, c4 = warp_sum_d(a2) / n;
                    if (kind == PB_FEAT_KURTOSIS) {
                        const double g2 = c4 / (c2 * c2 + 1e-10) - 3.0;
                        result = ((n - 1.0) / ((n - 2.0) * (n - 3.0) + 1e-10)) * ((n + 1.0) * g2 + 6.0);
                    } else {
                        const double g1 = c3 / (pow(c2, 1.5) + 1e-10);
                        result = g1 * sqrt(n * (n - 1.0)) / (n - 2.0 + 1e-10);
                    }
                } else if (kind == PB_FEAT_AUTOCORRELATION) {
                    const double ac = warp_sum_d(a1);
                    result = lag == 0 ? 1.0 : (lag >= nwin ? 0.0 : ac / (m2 + 1e-10));
                } else {
                    const double sd = sqrt(m2 / n);
                    double c = 0.0;
                    for (int i = lane; i < nwin; i += 32) c += fabs(static_cast<double>(x[i]) - mean) > param * sd;
                    result = warp_sum_d(c) / n;
                }
                break;
            }
            case PB_FEAT_ABS_SUM_CHANGES:
            case PB_FEAT_MEAN_ABS_CHANGE: {
                for (int i = lane + 1; i < nwin; i += 32) a0 += fabs(static_cast<double>(x[i]) - static_cast<double>(x[i - 1]));
                const double tot = warp_sum_d(a0);
                result = kind == PB_FEAT_ABS_SUM_CHANGES ? tot : tot / (n - 1.0);
                break;
            }
            case PB_FEAT_MEAN_CHANGE:
                result = (static_cast<double>(x[nwin - 1]) - static_cast<double>(x[0])) / (n - 1.0);
                break;
            case PB_FEAT_MEAN_SECOND_DERIV:
                result = nwin < 3 ? CUDART_NAN
                                  : (static_cast<double>(x[nwin - 1]) - static_cast<double>(x[nwin - 2]) -
                                     static_cast<double>(x[1]) + static_cast<double>(x[0])) /
                                        (2.0 * (n - 2.0));
                break;
            case PB_FEAT_COUNT_ABOVE_MEAN:
            case PB_FEAT_COUNT_BELOW_MEAN:
            case PB_FEAT_COUNT_ABOVE:
            case PB_FEAT_COUNT_BELOW: {
                const bool rel_mean = kind == PB_FEAT_COUNT_ABOVE_MEAN || kind == PB_FEAT_COUNT_BELOW_MEAN;
                const bool above = kind == PB_FEAT_COUNT_ABOVE_MEAN || kind == PB_FEAT_COUNT_ABOVE;
                const double level = rel_mean ? mean : param;
                for (int i = lane; i < nwin; i += 32) {
                    const double v = static_cast<double>(x[i]);
                    a0 += above ? (v > level) : (v < level);
                }
                const double c = warp_sum_d(a0);
                result = rel_mean ? c : c / n;
                break;
            }
            case PB_FEAT_NUMBER_PEAKS: {  // strict local maxima with support k on each side
                // consecutive indices per 32-wide batch, so the peak values of the
                // orbit data can be written in time order (ballot + prefix count)
                const int k = static_cast<int>(param);
                const int pi = plan.peak_idx[m];
                double* pk = (plan.peaks_out && pi >= 0)
                                 ? plan.peaks_out + (traj * plan.n_peak_cols + pi) * static_cast<int64_t>(plan.peak_cap)
                                 : nullptr;
                int count = 0;
                if (2 * k < nwin) {
                    for (int i0 = k; i0 < nwin - k; i0 += 32) {
                        const int i = i0 + lane;
                        bool peak = i < nwin - k;
                        if (peak) {
                            const float c = x[i];
                            for (int j = 1; j <= k && peak; ++j) peak = (c > x[i - j]) && (c > x[i + j]);
                        }
                        const unsigned mask = __ballot_sync(0xffffffffu, peak);
                        const int pos = count + __popc(mask & ((1u << lane) - 1u));
                        if (pk && peak && pos < plan.peak_cap) pk[pos] = static_cast<double>(x[i]);
                        count += __popc(mask);
                    }
                }
                if (pk)
                    for (int i = count + lane; i < plan.peak_cap; i += 32) pk[i] = CUDART_NAN;
                result = static_cast<double>(count);
                break;
            }
            case PB_FEAT_SPKT_WELCH:
            case PB_FEAT_FFT_REAL:
            case PB_FEAT_FFT_IMAG:
            case PB_FEAT_FFT_ABS:
            case PB_FEAT_FFT_ANGLE: {  // coefficient k of the one-sided DFT (rfft)
                const int k = static_cast<int>(param);
                if (k > nwin / 2) {
                    result = 0.0;  // past the last rfft coefficient
                    break;
                }
                for (int i = lane; i < nwin; i += 32) {
                    // phase k i / N in turns, reduced exactly in integers
                    const int64_t r = (static_cast<int64_t>(k) * i) % nwin;
                    double sn, cs;
                    sincospi(2.0 * static_cast<double>(r) / n, &sn, &cs);
                    const double v = static_cast<double>(x[i]);
                    a0 = fma(v, cs, a0);
                    a1 = fma(-v, sn, a1);
                }
                const double re = warp_sum_d(a0), im = warp_sum_d(a1);
                result = kind == PB_FEAT_FFT_REAL   ? re
                         : kind == PB_FEAT_FFT_IMAG ? im
                         : kind == PB_FEAT_FFT_ABS  ? hypot(re, im)
                         : kind == PB_FEAT_FFT_ANGLE ? atan2(im, re)
                                                     : (re * re + im * im) / n;  // power / N
                break;
            }
            case PB_FEAT_TREND_SLOPE:
            case PB_FEAT_TREND_INTERCEPT:
            case PB_FEAT_TREND_RVALUE:
            case PB_FEAT_TREND_PVALUE:
            case PB_FEAT_TREND_STDERR: {  // least squares of x on t = 0..N-1
                const double tm = 0.5 * (n - 1.0);
                for (int i = lane; i < nwin; i += 32) {
                    const double dt = static_cast<double>(i) - tm, dx = static_cast<double>(x[i]) - mean;
                    a0 += dt * dt;
                    a1 += dt * dx;
                    a2 += dx * dx;
                }
                const double ss_tt = warp_sum_d(a0), ss_tx = warp_sum_d(a1), ss_xx = warp_sum_d(a2);
                const double slope = ss_tx / (ss_tt + 1e-10);
                const double intercept = mean - slope * tm;
                const double r = ss_tx / (sqrt(ss_tt * ss_xx) + 1e-10);
                if (kind == PB_FEAT_TREND_SLOPE) {
                    result = slope;
                } else if (kind == PB_FEAT_TREND_INTERCEPT) {
                    result = intercept;
                } else if (kind == PB_FEAT_TREND_RVALUE) {
                    result = r;
                } else if (kind == PB_FEAT_TREND_PVALUE) {  // the reference's pseudo p-value
                    const double tstat = r * sqrt(n - 2.0) / (sqrt(1.0 - r * r) + 1e-10);
                    result = 1.0 / (1.0 + fabs(tstat));
                } else {
                    double rss = 0.0;
                    for (int i = lane; i < nwin; i += 32) {
                        const double e = static_cast<double>(x[i]) - (slope * static_cast<double>(i) + intercept);
                        rss += e * e;
                    }
                    result = sqrt(warp_sum_d(rss) / (n - 2.0) / (ss_tt + 1e-10));
                }
                break;
            }
            case PB_FEAT_FIRST_LOC_MAX:
            case PB_FEAT_FIRST_LOC_MIN:
            case PB_FEAT_LAST_LOC_MAX:
            case PB_FEAT_LAST_LOC_MIN: {  // index of the first (last) extreme / N
                const bool want_max = kind == PB_FEAT_FIRST_LOC_MAX || kind == PB_FEAT_LAST_LOC_MAX;
                const bool last = kind == PB_FEAT_LAST_LOC_MAX || kind == PB_FEAT_LAST_LOC_MIN;
                float best = want_max ? -CUDART_INF_F : CUDART_INF_F;
                int bi = -1;
                bool nan_seen = false;
                for (int i = lane; i < nwin; i += 32) {
                    const float v = x[i];
                    nan_seen |= isnan(v);
                    const bool better = want_max ? (v > best || (last && v == best)) : (v < best || (last && v == best));
                    if (bi < 0 || better) {
                        best = v;
                        bi = i;
                    }
                }
                for (int off = 16; off > 0; off >>= 1) {
                    const float ov = __shfl_down_sync(0xffffffffu, best, off);
                    const int oi = __shfl_down_sync(0xffffffffu, bi, off);
                    const bool take = oi >= 0 && (bi < 0 || (want_max ? ov > best : ov < best) ||
                                                  (ov == best && (last ? oi > bi : oi < bi)));
                    if (take) {
                        best = ov;
                        bi = oi;
                    }
                }
                bi = __shfl_sync(0xffffffffu, bi, 0);
                result = __any_sync(0xffffffffu, nan_seen) ? CUDART_NAN : static_cast<double>(bi) / n;
                break;
            }
            case PB_FEAT_CID_CE: {
                for (int i = lane; i < nwin; i += 32) {
                    const double dx = static_cast<double>(x[i]) - mean;
                    a1 += dx * dx;
                    if (i > 0) {
                        const double d = static_cast<double>(x[i]) - static_cast<double>(x[i - 1]);
                        a0 += d * d;
                    }
                }
                const double ce = sqrt(warp_sum_d(a0));
                const double sd = sqrt(warp_sum_d(a1) / n);
                result = param != 0.0 ? ce / (sd + 1e-10) : ce;
                break;
            }
            case PB_FEAT_LARGE_STD: {  // population std > r * range, as 1 / 0
                float mx = -CUDART_INF_F, mn = CUDART_INF_F;
                for (int i = lane; i < nwin; i += 32) {
                    const double d = static_cast<double>(x[i]) - mean;
                    a0 += d * d;
                    mx = fmaxf(mx, x[i]);
                    mn = fminf(mn, x[i]);
                }
                for (int off = 16; off > 0; off >>= 1) {
                    mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, off));
                    mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, off));
                }
                const double sd = sqrt(warp_sum_d(a0) / n);
                result = sd > param * (static_cast<double>(mx) - static_cast<double>(mn)) ? 1.0 : 0.0;
                break;
            }
            case PB_FEAT_INDEX_MASS_QUANTILE: {  // first index where cumsum |x| >= q * total, / N
                for (int i = lane; i < nwin; i += 32) a0 += fabs(static_cast<double>(x[i]));
                const double thr = param * warp_sum_d(a0);
                double carry = 0.0;
                int found = -1;
                for (int i0 = 0; i0 < nwin && found < 0; i0 += 32) {
                    const int i = i0 + lane;
                    double c = i < nwin ? fabs(static_cast<double>(x[i])) : 0.0;
                    for (int off = 1; off < 32; off <<= 1) {  // inclusive prefix sum
                        const double o = __shfl_up_sync(0xffffffffu, c, off);
                        if (lane >= off) c += o;
                    }
                    c += carry;
                    const unsigned hit = __ballot_sync(0xffffffffu, i < nwin && c >= thr);
                    if (hit) found = i0 + __ffs(hit) - 1;
                    carry = __shfl_sync(0xffffffffu, c, 31);
                }
                result = static_cast<double>(found < 0 ? 0 : found) / n;
                break;
            }
            case PB_FEAT_LONGEST_STRIKE_ABOVE:
            case PB_FEAT_LONGEST_STRIKE_BELOW: {  // longest run of samples above (below) the mean
                int run = 0, best = 0;  // run: length of the run ending at the previous chunk's end
                for (int i0 = 0; i0 < nwin; i0 += 32) {
                    const int i = i0 + lane;
                    const double v = i < nwin ? static_cast<double>(x[i]) : mean;
                    const bool on = i < nwin && (kind == PB_FEAT_LONGEST_STRIKE_ABOVE ? v > mean : v < mean);
                    const unsigned m = __ballot_sync(0xffffffffu, on);
                    // run ending at this lane: back to the last lane (at or below) that is off
                    const unsigned off_mask = ~m & ((lane == 31) ? 0xffffffffu : ((1u << (lane + 1)) - 1u));
                    const int here = !on ? 0 : (off_mask ? lane - (31 - __clz(off_mask)) : lane + 1 + run);
                    int mx = here;
                    for (int o = 16; o > 0; o >>= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
                    best = max(best, mx);
                    run = __shfl_sync(0xffffffffu, here, 31);
                }
                result = static_cast<double>(best);
                break;
            }
            case PB_FEAT_HAS_DUP_MAX:
            case PB_FEAT_HAS_DUP_MIN: {  // the extreme occurs more than once, as 1 / 0
                const bool want_max = kind == PB_FEAT_HAS_DUP_MAX;
                float e = want_max ? -CUDART_INF_F : CUDART_INF_F;
                bool nan_seen = false;
                for (int i = lane; i < nwin; i += 32) {
                    nan_seen |= isnan(x[i]);
                    e = want_max ? fmaxf(e, x[i]) : fminf(e, x[i]);
                }
                for (int off = 16; off > 0; off >>= 1) {
                    const float o = __shfl_xor_sync(0xffffffffu, e, off);
                    e = want_max ? fmaxf(e, o) : fminf(e, o);
                }
                int cnt = 0;
                for (int i = lane; i < nwin; i += 32) cnt += x[i] == e;
                for (int off = 16; off > 0; off >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, off);
                // torch.max propagates NaN, and NaN == NaN is false: no duplicate then
                result = (!__any_sync(0xffffffffu, nan_seen) && cnt > 1) ? 1.0 : 0.0;
                break;
            }
            case PB_FEAT_BINNED_ENTROPY: {  // entropy of max_bins equal-width bins over [min, max]
                const int bins = static_cast<int>(param);
                float mx = -CUDART_INF_F, mn = CUDART_INF_F;
                for (int i = lane; i < nwin; i += 32) {
                    mx = fmaxf(mx, x[i]);
                    mn = fminf(mn, x[i]);
                }
                for (int off = 16; off > 0; off >>= 1) {
                    mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, off));
                    mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, off));
                }
                if (mx == mn) {
                    result = 0.0;  // a constant window
                    break;
                }
                for (int b = lane; b < bins; b += 32) h[b] = 0u;
                __syncwarp();
                const double lo = mn, range = static_cast<double>(mx) - lo;
                for (int i = lane; i < nwin; i += 32) {
                    const double u = (static_cast<double>(x[i]) - lo) / (range + 1e-10) * (bins - 1e-6);
                    long long b = static_cast<long long>(u);  // truncation, as .long()
                    b = b < 0 ? 0 : (b > bins - 1 ? bins - 1 : b);
                    atomicAdd(&h[b], 1u);
                }
                __syncwarp();
                for (int b = lane; b < bins; b += 32) {
                    if (h[b] > 0u) {
                        const double p = fmax(static_cast<double>(h[b]) / n, 1e-10);
                        a0 -= p * log(p);
                    }
                }
                result = warp_sum_d(a0);
                break;
            }
            case PB_FEAT_MEAN_N_ABS_MAX: {  // mean of the k largest |x| (ties by index, as topk)
                const int k = min(static_cast<int>(param), nwin);
                float prev = CUDART_INF_F;
                int prev_i = -1;
                double tot = 0.0;
                for (int r = 0; r < k; ++r) {
                    // the largest (|x|, -index) strictly below the previous pick
                    float best = -1.f;
                    int bi = -1;
                    for (int i = lane; i < nwin; i += 32) {
                        const float v = fabsf(x[i]);
                        const bool below = v < prev || (v == prev && i > prev_i);
                        if (below && (bi < 0 || v > best)) {
                            best = v;
                            bi = i;
                        }
                    }
                    for (int off = 16; off > 0; off >>= 1) {
                        const float ov = __shfl_down_sync(0xffffffffu, best, off);
                        const int oi = __shfl_down_sync(0xffffffffu, bi, off);
                        if (oi >= 0 && (bi < 0 || ov > best || (ov == best && oi < bi))) {
                            best = ov;
                            bi = oi;
                        }
                    }
                    prev = __shfl_sync(0xffffffffu, best, 0);
                    prev_i = __shfl_sync(0xffffffffu, bi, 0);
                    tot += static_cast<double>(prev);
                }
                result = tot / k;
                break;
            }
            case PB_FEAT_BENFORD: {  // Pearson correlation of first-digit frequencies with Benford's law
                unsigned cnt[9];
#pragma unroll
                for (int dgt = 0; dgt < 9; ++dgt) cnt[dgt] = 0u;
                for (int i = lane; i < nwin; i += 32) {
                    const double v = fabs(static_cast<double>(x[i]));
                    if (v > 0.0) {
                        const double fl = floor(log10(v));
                        const long long dg = static_cast<long long>(floor(v / pow(10.0, fl)));
                        if (dg >= 1 && dg <= 9) {
#pragma unroll
                            for (int dgt = 0; dgt < 9; ++dgt) cnt[dgt] += (dg == dgt + 1) ? 1u : 0u;
                        }
                    }
                }
                double f[9], tot = 0.0;
#pragma unroll
                for (int dgt = 0; dgt < 9; ++dgt) {
                    unsigned c = cnt[dgt];
                    for (int off = 16; off > 0; off >>= 1) c += __shfl_xor_sync(0xffffffffu, c, off);
                    f[dgt] = static_cast<double>(c);
                    tot += f[dgt];
                }
                double fm = 0.0, bm = 0.0, b[9];
#pragma unroll
                for (int dgt = 0; dgt < 9; ++dgt) {
                    f[dgt] /= tot + 1e-10;
                    fm += f[dgt];
                    b[dgt] = log10(1.0 + 1.0 / (dgt + 1));
                    bm += b[dgt];
                }
                fm /= 9.0;
                bm /= 9.0;
                double sfb = 0.0, sff = 0.0, sbb = 0.0;
#pragma unroll
                for (int dgt = 0; dgt < 9; ++dgt) {
                    sfb += (f[dgt] - fm) * (b[dgt] - bm);
                    sff += (f[dgt] - fm) * (f[dgt] - fm);
                    sbb += (b[dgt] - bm) * (b[dgt] - bm);
                }
                // unbiased (n - 1 = 8) standard deviations, as torch.std
                const double corr = sfb / (sqrt(sff / 8.0) * sqrt(sbb / 8.0) * 9.0 + 1e-10);
                result = tot >= 10.0 ? corr : 0.0;
                break;
            }
            case PB_FEAT_C3:
            case PB_FEAT_TIME_REVERSAL: {
                const int lag = static_cast<int>(param);
                if (2 * static_cast<int64_t>(lag) >= nwin) {
                    result = 0.0;
                    break;
                }
                const int m3 = nwin - 2 * lag;
                for (int i = lane; i < m3; i += 32) {
                    const double x0 = x[i], x1 = x[i + lag], x2 = x[i + 2 * lag];
                    a0 += kind == PB_FEAT_C3 ? x0 * x1 * x2 : x2 * x2 * x1 - x1 * x0 * x0;
                }
                result = warp_sum_d(a0) / static_cast<double>(m3);
                break;
            }
            case PB_FEAT_VAR_LARGER_THAN_STD: {  // population std > 1, as 1 / 0
                for (int i = lane; i < nwin; i += 32) {
                    const double d = static_cast<double>(x[i]) - mean;
                    a0 += d * d;
                }
                result = sqrt(warp_sum_d(a0) / n) > 1.0 ? 1.0 : 0.0;
                break;
            }
            case PB_FEAT_PARTIAL_AUTOCORRELATION:
            case PB_FEAT_AGG_AUTOCORR_MEAN:
            case PB_FEAT_AGG_AUTOCORR_MEDIAN:
            case PB_FEAT_AGG_AUTOCORR_VAR: {
                // autocorrelations acf[k] = sum d_i d_(i+k) / (sum d_i^2 + 1e-10) for k = 1..ml,
                // one warp reduction per lag, kept in this warp's shared doubles
                const bool pacf = kind == PB_FEAT_PARTIAL_AUTOCORRELATION;
                const int want = static_cast<int>(param);
                if (pacf && want == 0) {
                    result = 1.0;
                    break;
                }
                const int ml = min(want, nwin - 1);
                if (ml < 1) {
                    result = pacf ? 0.0 : CUDART_NAN;
                    break;
                }
                double* hd = reinterpret_cast<double*>(h);  // acf[k] at hd[k - 1]; phi[k] at hd[63 + k]
                for (int i = lane; i < nwin; i += 32) {
                    const double d = static_cast<double>(x[i]) - mean;
                    a0 += d * d;
                }
                const double m2 = warp_sum_d(a0);
                for (int k = 1; k <= ml; ++k) {
                    double r = 0.0;
                    for (int i = lane; i + k < nwin; i += 32)
                        r += (static_cast<double>(x[i]) - mean) * (static_cast<double>(x[i + k]) - mean);
                    r = warp_sum_d(r);
                    if (lane == 0) hd[k - 1] = r / (m2 + 1e-10);
                }
                __syncwarp();
                if (pacf) {  // Durbin-Levinson on lane 0 (ml <= 63), the update in place by pairs (j, k - j)
                    if (lane == 0) {
                        double* phi = hd + 63;
                        phi[1] = hd[0];
                        for (int k = 2; k <= ml; ++k) {
                            double num = hd[k - 1], den = 1.0;
                            for (int j = 1; j < k; ++j) {
                                num -= phi[j] * hd[k - j - 1];
                                den -= phi[j] * hd[j - 1];
                            }
                            const double pk = num / (den + 1e-10);
                            for (int j = 1, l = k - 1; j <= l; ++j, --l) {
                                const double pj = phi[j], pl = phi[l];
                                phi[j] = pj - pk * pl;
                                if (l != j) phi[l] = pl - pk * pj;
                            }
                            phi[k] = pk;
                        }
                        result = want <= ml ? phi[want] : 0.0;
                    }
                    __syncwarp();
                    break;
                }
                double sa = 0.0;
                for (int k = lane; k < ml; k += 32) sa += hd[k];
                const double am = warp_sum_d(sa) / ml;
                if (kind == PB_FEAT_AGG_AUTOCORR_MEAN) {
                    result = am;
                } else if (kind == PB_FEAT_AGG_AUTOCORR_VAR) {  // population variance
                    double v = 0.0;
                    for (int k = lane; k < ml; k += 32) v += (hd[k] - am) * (hd[k] - am);
                    result = warp_sum_d(v) / ml;
                } else {  // lower median: the value with at most (ml-1)/2 smaller and more not larger
                    const int kk = (ml - 1) / 2;
                    double med = CUDART_NAN;
                    bool found = false;
                    for (int c = lane; c < ml; c += 32) {
                        const double v = hd[c];
                        int less = 0, leq = 0;
                        for (int q = 0; q < ml; ++q) {
                            less += hd[q] < v ? 1 : 0;
                            leq += hd[q] <= v ? 1 : 0;
                        }
                        if (less <= kk && kk < leq) {
                            med = v;
                            found = true;
                        }
                    }
                    const unsigned b = __ballot_sync(0xffffffffu, found);
                    med = __shfl_sync(0xffffffffu, med, b ? __ffs(b) - 1 : 0);
                    result = b ? med : CUDART_NAN;
                }
                __syncwarp();
                break;
            }
            case PB_FEAT_ENERGY_RATIO_BY_CHUNKS: {  // energy of chunk segment_focus of num_segments / total
                const int ns = static_cast<int>(param);
                const int size = nwin / ns;
                if (size == 0) {
                    result = 0.0;
                    break;
                }
                const int64_t start = static_cast<int64_t>(plan.param2[m]) * size;
                const int64_t end = min(start + size, static_cast<int64_t>(nwin));
                for (int i = lane; i < nwin; i += 32) {
                    const double v = static_cast<double>(x[i]);
                    a0 += v * v;
                    if (i >= start && i < end) a1 += v * v;
                }
                const double tot = warp_sum_d(a0);
                result = warp_sum_d(a1) / (tot + 1e-10);
                break;
            }
            case PB_FEAT_COUNT_IN_RANGE: {  // min_val <= x <= max_val, compared in the window's FP32
                const float lo = static_cast<float>(param), hi = static_cast<float>(plan.param2[m]);
                for (int i = lane; i < nwin; i += 32) a0 += (x[i] >= lo && x[i] <= hi) ? 1.0 : 0.0;
                result = warp_sum_d(a0);
                break;
            }
            case PB_FEAT_CHANGE_QUANTILES_MEAN:
            case PB_FEAT_CHANGE_QUANTILES_VAR:
            case PB_FEAT_CHANGE_QUANTILES_ABS_MEAN:
            case PB_FEAT_CHANGE_QUANTILES_ABS_VAR: {
                // changes between neighbours inside [quantile ql, quantile qh]: their mean or
                // population variance over the count (0 if none; a NaN leaves no corridor)
                bool nan_seen = false;
                for (int i = lane; i < nwin; i += 32) nan_seen |= isnan(x[i]);
                if (__any_sync(0xffffffffu, nan_seen)) {
                    result = 0.0;
                    break;
                }
                double qv[2];
                for (int e = 0; e < 2; ++e) {
                    const double pos = (e == 0 ? param : plan.param2[m]) * (nwin - 1);
                    const int lo = static_cast<int>(floor(pos));
                    const int hi = lo + 1 < nwin ? lo + 1 : nwin - 1;
                    const double va = select_rank(x, nwin, static_cast<unsigned>(lo), h, lane);
                    const double vb = hi == lo ? va : select_rank(x, nwin, static_cast<unsigned>(hi), h, lane);
                    qv[e] = va + (vb - va) * (pos - lo);
                }
                const bool isabs = kind == PB_FEAT_CHANGE_QUANTILES_ABS_MEAN || kind == PB_FEAT_CHANGE_QUANTILES_ABS_VAR;
                const bool is_var = kind == PB_FEAT_CHANGE_QUANTILES_VAR || kind == PB_FEAT_CHANGE_QUANTILES_ABS_VAR;
                for (int i = lane + 1; i < nwin; i += 32) {
                    const double p = static_cast<double>(x[i - 1]), c = static_cast<double>(x[i]);
                    if (p >= qv[0] && p <= qv[1] && c >= qv[0] && c <= qv[1]) {
                        a0 += isabs ? fabs(c - p) : c - p;
                        a1 += 1.0;
                    }
                }
                const double cnt = warp_sum_d(a1);
                const double mu = warp_sum_d(a0) / cnt;
                if (cnt == 0.0) {
                    result = 0.0;
                } else if (!is_var) {
                    result = mu;
                } else {
                    for (int i = lane + 1; i < nwin; i += 32) {
                        const double p = static_cast<double>(x[i - 1]), c = static_cast<double>(x[i]);
                        if (p >= qv[0] && p <= qv[1] && c >= qv[0] && c <= qv[1]) {
                            const double d = (isabs ? fabs(c - p) : c - p) - mu;
                            a2 += d * d;
                        }
                    }
                    result = warp_sum_d(a2) / cnt;
                }
                break;
            }
            case PB_FEAT_ACF_PERIOD_STRENGTH:
            case PB_FEAT_ACF_PERIOD_LAG: {
                // first autocorrelation peak (midpoint of a maximal run of equal values
                // entered from below and left downwards) at lag >= min_lag above the
                // threshold: its value or its lag, else 0.  acf[k] = r_k / (r_0 + 1e-10)
                // of the window centred and scaled by its unbiased std + 1e-10.  Lags
                // are computed 32 at a time (one per lane, each a sequential sum) and
                // scanned in order by every lane alike; the scan stops at the peak.
                if (nwin < 2) {
                    result = 0.0;
                    break;
                }
                const int min_lag = static_cast<int>(param);
                const double thr = plan.param2[m];
                for (int i = lane; i < nwin; i += 32) {
                    const double d = static_cast<double>(x[i]) - mean;
                    a0 += d * d;
                }
                const double m2 = warp_sum_d(a0);
                const double sd = sqrt(m2 / (n - 1.0)) + 1e-10, ss = sd * sd;
                const double r0 = m2 / ss, den = r0 + 1e-10;
                double v_run = r0 / den;  // the run holding lag 0 is never a peak
                int run_a = 0;
                bool rose = false, found = false;
                double out_v = 0.0, out_lag = 0.0;
                for (int k0 = 1; k0 < nwin && !found; k0 += 32) {
                    const int k = k0 + lane;
                    double r = 0.0;
                    for (int i = 0; i + k < nwin; ++i)
                        r += (static_cast<double>(x[i]) - mean) * (static_cast<double>(x[i + k]) - mean);
                    const double val = (r / ss) / den;
                    const int cnt = min(32, nwin - k0);
                    for (int j = 0; j < cnt; ++j) {
                        const double v = __shfl_sync(0xffffffffu, val, j);
                        if (v == v_run) continue;
                        if (rose && v < v_run) {
                            const int mid = (run_a + k0 + j - 1) / 2;
                            if (mid >= min_lag && v_run > thr) {
                                found = true;
                                out_v = v_run;
                                out_lag = static_cast<double>(mid);
                                break;
                            }
                        }
                        rose = v_run < v;
                        run_a = k0 + j;
                        v_run = v;
                    }
                }
                result = kind == PB_FEAT_ACF_PERIOD_STRENGTH ? out_v : out_lag;
                break;
            }
            case PB_FEAT_AGG_TREND_MEAN:
            case PB_FEAT_AGG_TREND_VAR:
            case PB_FEAT_AGG_TREND_MIN:
            case PB_FEAT_AGG_TREND_MAX: {
                // linear trend of chunk aggregates (a partial last chunk dropped), each
                // chunk aggregated sequentially by the lane that needs it
                const int cs = static_cast<int>(param), nc = nwin / cs;
                if (nc < 2) {
                    result = 0.0;
                    break;
                }
                const auto agg = [&](int c) -> double {
                    const float* q = x + static_cast<int64_t>(c) * cs;
                    double s1 = 0.0, lo = q[0], hi = q[0];
                    for (int i = 0; i < cs; ++i) {
                        const double v = static_cast<double>(q[i]);
                        s1 += v;
                        lo = v < lo ? v : lo;
                        hi = v > hi ? v : hi;
                    }
                    const double cm = s1 / cs;
                    if (kind == PB_FEAT_AGG_TREND_MEAN) return cm;
                    if (kind == PB_FEAT_AGG_TREND_MIN) return lo;
                    if (kind == PB_FEAT_AGG_TREND_MAX) return hi;
                    double v2 = 0.0;
                    for (int i = 0; i < cs; ++i) v2 += (static_cast<double>(q[i]) - cm) * (static_cast<double>(q[i]) - cm);
                    return v2 / cs;
                };
                result = warp_trend(agg, nc, static_cast<int>(plan.param2[m]), lane);
                break;
            }
            case PB_FEAT_AR_COEFFICIENT: {
                // Yule-Walker: R phi = r, R_ij = acf[|i-j|] + 1e-6 delta_ij, r = acf[1..k];
                // acf by warp reductions into this warp's shared doubles (R at [0, 110),
                // acf at [110, 121)), elimination with partial pivoting on lane 0
                const int k = static_cast<int>(param), coeff = static_cast<int>(plan.param2[m]);
                if (coeff >= k) {
                    result = 0.0;
                    break;
                }
                double* hd = reinterpret_cast<double*>(h);
                double* acf = hd + 110;
                for (int i = lane; i < nwin; i += 32) {
                    const double d = static_cast<double>(x[i]) - mean;
                    a0 += d * d;
                }
                const double m2 = warp_sum_d(a0);
                for (int l = 1; l <= k; ++l) {
                    double r = 0.0;
                    for (int i = lane; i + l < nwin; i += 32)
                        r += (static_cast<double>(x[i]) - mean) * (static_cast<double>(x[i + l]) - mean);
                    r = warp_sum_d(r);
                    if (lane == 0) acf[l] = r / (m2 + 1e-10);
                }
                if (lane == 0) {
                    acf[0] = m2 / (m2 + 1e-10);
                    double* R = hd;  // k rows of k + 1 (the last column: r, then phi)
                    for (int i = 0; i < k; ++i) {
                        for (int j = 0; j < k; ++j) R[i * 11 + j] = acf[abs(i - j)] + (i == j ? 1e-6 : 0.0);
                        R[i * 11 + k] = acf[i + 1];
                    }
                    for (int c = 0; c < k; ++c) {
                        int piv = c;
                        for (int i = c + 1; i < k; ++i)
                            if (fabs(R[i * 11 + c]) > fabs(R[piv * 11 + c])) piv = i;
                        if (piv != c)
                            for (int j = 0; j <= k; ++j) {
                                const double t = R[c * 11 + j];
                                R[c * 11 + j] = R[piv * 11 + j];
                                R[piv * 11 + j] = t;
                            }
                        for (int i = c + 1; i < k; ++i) {
                            const double f = R[i * 11 + c] / R[c * 11 + c];
                            for (int j = c; j <= k; ++j) R[i * 11 + j] -= f * R[c * 11 + j];
                        }
                    }
                    for (int i = k - 1; i >= 0; --i) {
                        double t = R[i * 11 + k];
                        for (int j = i + 1; j < k; ++j) t -= R[i * 11 + j] * R[j * 11 + k];
                        R[i * 11 + k] = t / R[i * 11 + i];
                    }
                    result = R[coeff * 11 + k];
                }
                __syncwarp();
                break;
            }
            case PB_FEAT_CWT: {
                // Ricker wavelet of width w correlated with the window padded by 4w
                // samples (reflected without the edge, or replicated when nwin < 4w), at
                // output index coeff; the prefactor rounded in FP32 as the reference forms it
                const int wd = static_cast<int>(param), coeff = static_cast<int>(plan.param2[m]);
                if (coeff < 0 || coeff >= nwin) {
                    result = 0.0;
                    break;
                }
                const float pref32 = __fdiv_rn(2.0f, __fmul_rn(__fsqrt_rn(static_cast<float>(3.0 * wd)),
                                                               static_cast<float>(1.3313353638003897)));
                const double pref = static_cast<double>(pref32), sig = static_cast<double>(wd);
                const int pad = 4 * wd;
                for (int j = lane; j <= 8 * wd; j += 32) {
                    const double t = static_cast<double>(j - pad);
                    const double psi = pref * (1.0 - (t / sig) * (t / sig)) * exp(-(t * t) / (2.0 * sig * sig));
                    int64_t q = static_cast<int64_t>(coeff) + j - pad;
                    if (nwin >= pad) {
                        if (q < 0) q = -q;
                        if (q >= nwin) q = 2ll * (nwin - 1) - q;
                    } else {
                        q = q < 0 ? 0 : (q >= nwin ? nwin - 1 : q);
                    }
                    a0 += static_cast<double>(x[q]) * psi;
                }
                result = warp_sum_d(a0);
                break;
            }
            case PB_FEAT_FRIEDRICH:
            case PB_FEAT_LANGEVIN: {
                // velocity v_i = x_(i+1) - x_i fitted by a degree-m polynomial of the
                // position x_i: the regularised normal equations (V'V + 1e-6 I) c = V'v from
                // warp sums of powers, solved on lane 0 (in this warp's shared doubles)
                const int deg = static_cast<int>(param);
                if (nwin < 2) {
                    result = 0.0;
                    break;
                }
                double S[13], T[7];
#pragma unroll
                for (int q = 0; q < 13; ++q) S[q] = 0.0;
#pragma unroll
                for (int q = 0; q < 7; ++q) T[q] = 0.0;
                for (int i = lane; i + 1 < nwin; i += 32) {
                    const double p = static_cast<double>(x[i]), v = static_cast<double>(x[i + 1]) - p;
                    double pw = 1.0;
#pragma unroll
                    for (int q = 0; q < 13; ++q) {
                        if (q <= 2 * deg) S[q] += pw;
                        if (q <= deg) T[q] += pw * v;
                        pw *= p;
                    }
                }
#pragma unroll
                for (int q = 0; q < 13; ++q) S[q] = warp_sum_d(S[q]);
#pragma unroll
                for (int q = 0; q < 7; ++q) T[q] = warp_sum_d(T[q]);
                double* A = reinterpret_cast<double*>(h);  // (deg + 1) rows of stride 8; column deg + 1: rhs, then c
                const int k = deg + 1;
                if (lane == 0) {
                    for (int r = 0; r < k; ++r) {
                        for (int c = 0; c < k; ++c) A[r * 8 + c] = S[2 * deg - r - c] + (r == c ? 1e-6 : 0.0);
                        A[r * 8 + k] = T[deg - r];
                    }
                    for (int col = 0; col < k; ++col) {
                        int piv = col;
                        for (int i = col + 1; i < k; ++i)
                            if (fabs(A[i * 8 + col]) > fabs(A[piv * 8 + col])) piv = i;
                        if (piv != col)
                            for (int j = 0; j <= k; ++j) {
                                const double t = A[col * 8 + j];
                                A[col * 8 + j] = A[piv * 8 + j];
                                A[piv * 8 + j] = t;
                            }
                        for (int i = col + 1; i < k; ++i) {
                            const double f = A[i * 8 + col] / A[col * 8 + col];
                            for (int j = col; j <= k; ++j) A[i * 8 + j] -= f * A[col * 8 + j];
                        }
                    }
                    for (int i = k - 1; i >= 0; --i) {
                        double t = A[i * 8 + k];
                        for (int j = i + 1; j < k; ++j) t -= A[i * 8 + j] * A[j * 8 + k];
                        A[i * 8 + k] = t / A[i * 8 + i];
                    }
                }
                __syncwarp();
                if (kind == PB_FEAT_FRIEDRICH) {
                    const int coeff = static_cast<int>(plan.param2[m]);
                    result = coeff <= deg ? A[coeff * 8 + k] : 0.0;
                } else {  // the largest position x_i (i < n-2) where the fit changes sign to i+1
                    double best = -CUDART_INF;
                    for (int i = lane; i + 2 < nwin; i += 32) {
                        const double p0 = static_cast<double>(x[i]), p1 = static_cast<double>(x[i + 1]);
                        double f0 = 0.0, f1 = 0.0;
                        for (int q = 0; q <= deg; ++q) {
                            f0 = f0 * p0 + A[q * 8 + k];
                            f1 = f1 * p1 + A[q * 8 + k];
                        }
                        if (f0 * f1 < 0.0) best = fmax(best, p0);
                    }
                    for (int off = 16; off > 0; off >>= 1) best = fmax(best, __shfl_xor_sync(0xffffffffu, best, off));
                    result = best == -CUDART_INF ? 0.0 : best;
                }
                __syncwarp();
                break;
            }
            case PB_FEAT_ADF_TESTSTAT:
            case PB_FEAT_ADF_PVALUE:
            case PB_FEAT_ADF_USEDLAG: {  // first difference regressed on the lagged value (usedlag: 1)
                if (kind == PB_FEAT_ADF_USEDLAG) {
                    result = 1.0;
                    break;
                }
                const int nm = nwin - 1;
                for (int i = lane; i < nm; i += 32) {
                    const double p = static_cast<double>(x[i]);
                    a0 += p;
                    a1 += static_cast<double>(x[i + 1]) - p;
                }
                const double xm = warp_sum_d(a0) / nm, ym = warp_sum_d(a1) / nm;
                a0 = 0.0;
                a1 = 0.0;
                for (int i = lane; i < nm; i += 32) {
                    const double p = static_cast<double>(x[i]), d = static_cast<double>(x[i + 1]) - p;
                    a0 += (p - xm) * (p - xm);
                    a1 += (p - xm) * (d - ym);
                }
                const double sxx = warp_sum_d(a0), sxy = warp_sum_d(a1);
                const double beta = sxy / (sxx + 1e-10);
                for (int i = lane; i < nm; i += 32) {
                    const double p = static_cast<double>(x[i]), d = static_cast<double>(x[i + 1]) - p;
                    const double e = d - (ym + beta * (p - xm));
                    a2 += e * e;
                }
                const double se = sqrt(warp_sum_d(a2) / (n - 3.0)) / (sqrt(sxx) + 1e-10);
                const double t = beta / (se + 1e-10);
                result = kind == PB_FEAT_ADF_TESTSTAT ? t : 1.0 / (1.0 + fabs(t));
                break;
            }
            case PB_FEAT_NUMBER_CWT_PEAKS: {
                // samples equal to the maximum of their +-width neighbourhood (a NaN in it
                // rules the sample out, as max pooling propagates NaN), for each width
                // 1..max_width with 2 width < n, averaged over those widths
                const int mw = static_cast<int>(param);
                int nw = 0;
                for (int wd = 1; wd <= mw; ++wd) {
                    if (!(2 * wd < nwin)) continue;
                    ++nw;
                    for (int i = wd + lane; i < nwin - wd; i += 32) {
                        const float xi = x[i];
                        bool nan_in = false, peak = true;
                        for (int j = i - wd; j <= i + wd; ++j) {
                            const float v = x[j];
                            nan_in |= isnan(v);
                            peak &= !(v > xi);
                        }
                        a0 += (peak && !nan_in) ? 1.0 : 0.0;
                    }
                }
                result = nw > 0 ? warp_sum_d(a0) / nw : 0.0;
                break;
            }
            case PB_FEAT_COUNT_VALUE: {  // samples equal to the value, compared in the window's FP32
                const float v = static_cast<float>(param);
                for (int i = lane; i < nwin; i += 32) a0 += x[i] == v ? 1.0 : 0.0;
                result = warp_sum_d(a0);
                break;
            }
            default: break;
        }
    }
    if (lane == 0) out[traj * n_features + col] = result;
}

// Block-wide FP64 sum over 256 threads (every thread gets the total).
__device__ double block_sum_d(double v, double* red)
{
    v = warp_sum_d(v);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = 0.0;
    for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) t += red[w];
    __syncthreads();
    return t;
}

// Block-wide argmax of psd[k] over k in [0, nb) with |k - skip| >= 2 (skip < 0:
// none), ties to the lower index; every thread gets the index (-1 if none).
__device__ int block_argmax(const double* psd, int nb, int skip, double* red, int* redi)
{
    double bv = -CUDART_INF;
    int bi = -1;
    for (int k = threadIdx.x; k < nb; k += blockDim.x) {
        if (skip >= 0 && abs(k - skip) < 2) continue;
        if (bi < 0 || psd[k] > bv) {
            bv = psd[k];
            bi = k;
        }
    }
    for (int off = 16; off > 0; off >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, bv, off);
        const int oi = __shfl_xor_sync(0xffffffffu, bi, off);
        if (oi >= 0 && (bi < 0 || ov > bv || (ov == bv && oi < bi))) {
            bv = ov;
            bi = oi;
        }
    }
    if ((threadIdx.x & 31) == 0) {
        red[threadIdx.x >> 5] = bv;
        redi[threadIdx.x >> 5] = bi;
    }
    __syncthreads();
    bv = -CUDART_INF;
    bi = -1;
    for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w)
        if (redi[w] >= 0 && (bi < 0 || red[w] > bv || (red[w] == bv && redi[w] < bi))) {
            bv = red[w];
            bi = redi[w];
        }
    __syncthreads();
    return bi;
}

// Power spectrum of the window (kinds 79..83): one 256-thread block per
// (trajectory, spectral column).  |X_k|^2 of the one-sided DFT, k = 0..n/2, by
// Goertzel recurrences in FP64 (four bins per thread per pass over the window,
// which every thread reads alike), closed as X_k = s1 - e^(-i w) s2; the spectrum
// stays in shared memory for the reductions: spectral_frequency_ratio (centred
// window, bin 0 zeroed; the two strongest bins at least two apart, ties to the
// lower index) and fft_aggregated (moments of the bin index under the normalised
// spectrum of the uncentred window).
__global__ void __launch_bounds__(256) k_window_spectrum(const float* __restrict__ win, int nwin, MedianPlan plan,
                                                         double* __restrict__ out, int n_features)
{
    extern __shared__ double psd[];  // nwin / 2 + 1 entries
    __shared__ double red[8];
    __shared__ int redi[8];
    const int64_t blk = blockIdx.x;
    const int64_t traj = blk / plan.n_spectral;
    const int m = plan.spectral_m[blk - traj * plan.n_spectral];
    const int kind = plan.kind[m];
    const float* x = win + (traj * plan.n_med + m) * static_cast<int64_t>(nwin);
    const int nb = nwin / 2 + 1;
    double sx = 0.0;
    for (int i = threadIdx.x; i < nwin; i += blockDim.x) sx += static_cast<double>(x[i]);
    const double shift = kind == PB_FEAT_SPECTRAL_FREQ_RATIO ? block_sum_d(sx, red) / nwin : 0.0;
    for (int k0 = 4 * threadIdx.x; k0 < nb; k0 += 4 * blockDim.x) {
        double c[4], sn[4], cs[4], s1[4], s2[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int k = min(k0 + j, nb - 1);
            sincospi(2.0 * static_cast<double>(k) / nwin, &sn[j], &cs[j]);
            c[j] = 2.0 * cs[j];
            s1[j] = 0.0;
            s2[j] = 0.0;
        }
        for (int i = 0; i < nwin; ++i) {
            const double v = static_cast<double>(x[i]) - shift;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const double t = fma(c[j], s1[j], v - s2[j]);
                s2[j] = s1[j];
                s1[j] = t;
            }
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            if (k0 + j >= nb) break;
            const double re = s1[j] - cs[j] * s2[j], im = sn[j] * s2[j];
            psd[k0 + j] = re * re + im * im;
        }
    }
    __syncthreads();
    double result;
    if (kind == PB_FEAT_FOURIER_ENTROPY) {  // shares clamped at 1e-10
        double a = 0.0;
        for (int k = threadIdx.x; k < nb; k += blockDim.x) a += psd[k];
        const double tot = block_sum_d(a, red) + 1e-10;
        a = 0.0;
        for (int k = threadIdx.x; k < nb; k += blockDim.x) {
            const double p = fmax(psd[k] / tot, 1e-10);
            a -= p * log(p);
        }
        result = block_sum_d(a, red);
    } else if (kind == PB_FEAT_SPECTRAL_FREQ_RATIO) {
        if (threadIdx.x == 0) psd[0] = 0.0;
        __syncthreads();
        const int first = block_argmax(psd, nb, -1, red, redi);
        result = 0.0;
        if (first >= 0 && !(psd[first] < 1e-10)) {
            const int second = block_argmax(psd, nb, first, red, redi);
            if (second >= 0 && first > 0) result = static_cast<double>(second) / first;
        }
    } else {
        double a = 0.0;
        for (int k = threadIdx.x; k < nb; k += blockDim.x) a += psd[k];
        const double tot = block_sum_d(a, red) + 1e-10;
        a = 0.0;
        for (int k = threadIdx.x; k < nb; k += blockDim.x) a += k * (psd[k] / tot);
        const double cen = block_sum_d(a, red);
        double v2 = 0.0, v3 = 0.0, v4 = 0.0;
        for (int k = threadIdx.x; k < nb; k += blockDim.x) {
            const double p = psd[k] / tot, d = k - cen;
            v2 += d * d * p;
            v3 += d * d * d * p;
            v4 += d * d * d * d * p;
        }
        const double var = block_sum_d(v2, red);
        const double m3 = block_sum_d(v3, red);
        const double m4 = block_sum_d(v4, red);
        if (kind == PB_FEAT_FFT_AGG_CENTROID) result = cen;
        else if (kind == PB_FEAT_FFT_AGG_VARIANCE) result = var;
        else if (kind == PB_FEAT_FFT_AGG_SKEW) result = m3 / (pow(var, 1.5) + 1e-10);
        else result = m4 / (var * var + 1e-10);
    }
    if (threadIdx.x == 0) out[traj * n_features + plan.col[m]] = result;
}

// Block-wide FP64 maximum over 256 threads (every thread gets it).
__device__ double block_max_d(double v, double* red)
{
    for (int off = 16; off > 0; off >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, off));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = -CUDART_INF;
    for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) t = fmax(t, red[w]);
    __syncthreads();
    return t;
}

__constant__ int kFactorial[8] = {1, 1, 2, 6, 24, 120, 720, 5040};

// Symbolic kinds (85, 86): one 256-thread block per (trajectory, column).
// permutation_entropy: every embedded vector (x_i, x_(i+tau), ..) gets the id
// sum_p idx[p] (d-1-p)!, idx the indices that sort it (ties in index order; the
// reference's id, which is not one-to-one on permutations), counted in a shared
// histogram of d! bins; the entropy of the id frequencies over log d!.
// lempel_ziv_complexity: the window is cut into `bins` equal bins over [min, max +
// 1e-10) and parsed into phrases, each the shortest substring from the current
// position that is not an earlier phrase; every phrase extends an earlier one by a
// symbol, so the phrases form a trie, held as an open-addressing table (node *
// 256 + symbol -> child) in shared memory and walked by one thread; the phrase
// count over n / log n.
__global__ void __launch_bounds__(256) k_window_symbolic(const float* __restrict__ win, int nwin, int table_size,
                                                         MedianPlan plan, double* __restrict__ out, int n_features)
{
    extern __shared__ __align__(16) unsigned sm[];
    __shared__ double red[8];
    const int64_t blk = blockIdx.x;
    const int64_t traj = blk / plan.n_symbolic;
    const int m = plan.symbolic_m[blk - traj * plan.n_symbolic];
    const int kind = plan.kind[m];
    const float* x = win + (traj * plan.n_med + m) * static_cast<int64_t>(nwin);
    double result = 0.0;
    if (kind == PB_FEAT_CORR_DIM) {
        // correlation_dimension: delay vectors of emb samples `lag` apart from the
        // window (kept as floats in shared memory); n_rvals radii between 0.1 and 0.5
        // unbiased std on a log scale, formed in FP32 as the reference's type promotion
        // does; every unordered pair of vectors adds 2 to the count of the smallest
        // radius it lies within (binary search, a shared histogram per warp); then
        // the least-squares slope of log C(r) on log r in centred form on thread 0
        const int emb = static_cast<int>(plan.param[m]), packed = static_cast<int>(plan.param2[m]);
        const int lag = packed / 1024, nr = packed % 1024;
        const int64_t M = static_cast<int64_t>(nwin) - static_cast<int64_t>(emb - 1) * lag;
        double sx = 0.0;
        for (int i = threadIdx.x; i < nwin; i += blockDim.x) sx += static_cast<double>(x[i]);
        const double mean = block_sum_d(sx, red) / nwin;
        double sv = 0.0;
        for (int i = threadIdx.x; i < nwin; i += blockDim.x) {
            const double d = static_cast<double>(x[i]) - mean;
            sv += d * d;
        }
        const double sd = sqrt(block_sum_d(sv, red) / (nwin - 1.0));
        result = CUDART_NAN;
        if (M >= 2) {
            float* wx = reinterpret_cast<float*>(sm);
            double* rv = reinterpret_cast<double*>(sm + (nwin + 3) / 4 * 4);
            unsigned* hist = reinterpret_cast<unsigned*>(rv + nr);
            const int nwarp = static_cast<int>(blockDim.x >> 5), warp = static_cast<int>(threadIdx.x >> 5);
            for (int i = threadIdx.x; i < nwin; i += blockDim.x) wx[i] = x[i];
            const double lmin = log(0.1 * sd + 1e-10), lmax = log(0.5 * sd + 1e-10);
            const float ld = static_cast<float>(lmax - lmin), lmin32 = static_cast<float>(lmin);
            const float step = nr > 1 ? __fdiv_rn(1.0f, static_cast<float>(nr - 1)) : 0.0f;
            for (int k = threadIdx.x; k < nr; k += blockDim.x) {
                const float a = k < nr / 2 ? __fmaf_rn(step, static_cast<float>(k), 0.0f)
                                           : __fmaf_rn(-step, static_cast<float>(nr - 1 - k), 1.0f);
                const float arg = __fadd_rn(lmin32, __fmul_rn(a, ld));
                rv[k] = static_cast<double>(static_cast<float>(exp(static_cast<double>(arg))));
            }
            for (int q = threadIdx.x; q < nwarp * nr; q += blockDim.x) hist[q] = 0u;
            __syncthreads();
            const double rmax = rv[nr - 1];
            for (int64_t i = threadIdx.x; i < M; i += blockDim.x) {
                float vi[16];
                for (int e = 0; e < emb; ++e) vi[e] = wx[i + static_cast<int64_t>(e) * lag];
                for (int64_t j = i + 1; j < M; ++j) {
                    double d2 = 0.0;
                    for (int e = 0; e < emb; ++e) {
                        const double df =
                            static_cast<double>(vi[e]) - static_cast<double>(wx[j + static_cast<int64_t>(e) * lag]);
                        d2 += df * df;
                    }
                    const double dist = sqrt(d2);
                    if (!(dist <= rmax)) continue;
                    int lo = 0, hi = nr - 1;  // smallest k with dist <= rv[k]
                    while (lo < hi) {
                        const int mid = (lo + hi) >> 1;
                        if (dist <= rv[mid]) hi = mid;
                        else lo = mid + 1;
                    }
                    atomicAdd(&hist[warp * nr + lo], 1u);
                }
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                const double pairs = static_cast<double>(M) * static_cast<double>(M - 1);
                double acc = 0.0, nv = 0.0, sr = 0.0, sc = 0.0;
                for (int k = 0; k < nr; ++k) {
                    for (int w = 0; w < nwarp; ++w) acc += 2.0 * hist[w * nr + k];
                    const double c = acc / pairs;
                    if (!(c > 0.0)) continue;
                    nv += 1.0;
                    sr += log(rv[k]);
                    sc += log(c + 1e-30);
                }
                double srr = 0.0, src = 0.0;
                acc = 0.0;
                for (int k = 0; k < nr; ++k) {
                    for (int w = 0; w < nwarp; ++w) acc += 2.0 * hist[w * nr + k];
                    const double c = acc / pairs;
                    if (!(c > 0.0)) continue;
                    const double dr = log(rv[k]) - sr / nv, dc = log(c + 1e-30) - sc / nv;
                    srr += dr * dr;
                    src += dr * dc;
                }
                const double den = nv * srr;
                result = (nv >= 2.0 && fabs(den) > 1e-10) ? (nv * src) / den : CUDART_NAN;
            }
        }
    } else if (kind == PB_FEAT_LYAP_R) {
        // lyapunov_r (Rosenstein): min_tsep from the mean frequency of the window's
        // spectrum zero-padded to 2n-1 (Goertzel per bin, bins over threads); each of
        // the first ntraj delay vectors takes the first nearest one more than min_tsep
        // away (threads over vectors, the window as floats in shared memory); the mean
        // log divergence at each step k (block sums), rounded to FP32 as the reference
        // stores it; the line fit on thread 0
        const int emb = static_cast<int>(plan.param[m]) / 1024, L = static_cast<int>(plan.param[m]) % 1024;
        const int lag = static_cast<int>(plan.param2[m]);
        const int64_t M = static_cast<int64_t>(nwin) - static_cast<int64_t>(emb - 1) * lag;
        result = CUDART_NAN;
        if (M >= 1) {
            float* wx = reinterpret_cast<float*>(sm);
            int* nb = reinterpret_cast<int*>(sm + (nwin + 3) / 4 * 4);
            for (int i = threadIdx.x; i < nwin; i += blockDim.x) wx[i] = x[i];
            __syncthreads();
            const int64_t N2 = 2ll * nwin - 1;
            double afp = 0.0, ap = 0.0;
            for (int64_t k = 1 + threadIdx.x; k <= N2 / 2; k += blockDim.x) {
                double sn, cs;
                sincospi(2.0 * static_cast<double>(k) / static_cast<double>(N2), &sn, &cs);
                const double c = 2.0 * cs;
                double s1 = 0.0, s2 = 0.0;
                for (int i = 0; i < nwin; ++i) {
                    const double t = fma(c, s1, static_cast<double>(wx[i]) - s2);
                    s2 = s1;
                    s1 = t;
                }
                const double re = s1 - cs * s2, im = sn * s2, p = re * re + im * im;
                afp += (static_cast<double>(k) / static_cast<double>(N2)) * p;
                ap += p;
            }
            const double sfp = block_sum_d(afp, red), sp = block_sum_d(ap, red);
            int64_t tsep = static_cast<int64_t>(ceil(1.0 / (sfp / (sp + 1e-10) + 1e-10)));
            const int64_t maxt = static_cast<int64_t>(0.25 * nwin);
            tsep = tsep > maxt ? maxt : tsep;
            tsep = tsep < 1 ? 1 : tsep;
            const int64_t ntraj = M - L + 1 > 1 ? M - L + 1 : 1;
            const auto dist = [&](int64_t a, int64_t b) -> double {
                if ((a > b ? a - b : b - a) <= tsep) return CUDART_INF;
                double d2 = 0.0;
                for (int e = 0; e < emb; ++e) {
                    const double df = static_cast<double>(wx[a + static_cast<int64_t>(e) * lag]) -
                                      static_cast<double>(wx[b + static_cast<int64_t>(e) * lag]);
                    d2 += df * df;
                }
                return sqrt(d2);
            };
            for (int64_t i = threadIdx.x; i < ntraj; i += blockDim.x) {
                double best = CUDART_INF;
                int bj = 0;
                for (int64_t j = 0; j < ntraj; ++j) {
                    const double d = dist(i, j);
                    if (d < best) {
                        best = d;
                        bj = static_cast<int>(j);
                    }
                }
                nb[i] = bj;
            }
            __syncthreads();
            double nf = 0.0, sk = 0.0, sd = 0.0, skk = 0.0, skd = 0.0;
            for (int k = 0; k < L; ++k) {
                double acc = 0.0, cnt = 0.0;
                for (int64_t i = threadIdx.x; i < ntraj; i += blockDim.x) {
                    if (i + k >= M || nb[i] + k >= M) continue;
                    const double d = dist(i + k, nb[i] + k);
                    if (!(d > 0.0)) continue;
                    acc += log(d);
                    cnt += 1.0;
                }
                acc = block_sum_d(acc, red);
                cnt = block_sum_d(cnt, red);
                const double div = static_cast<double>(static_cast<float>(cnt > 0.0 ? acc / cnt : CUDART_NAN));
                if (!isfinite(div)) continue;
                nf += 1.0;
                sk += k;
                sd += div;
                skk += static_cast<double>(k) * k;
                skd += k * div;
            }
            const double den = nf * skk - sk * sk;
            result = (nf >= 2.0 && fabs(den) > 1e-10) ? (nf * skd - sk * sd) / den : CUDART_NAN;
        }
    } else if (kind == PB_FEAT_PERMUTATION_ENTROPY) {
        const int tau = static_cast<int>(plan.param[m]), d = static_cast<int>(plan.param2[m]);
        const int64_t npat = static_cast<int64_t>(nwin) - static_cast<int64_t>(d - 1) * tau;
        if (npat > 0) {
            const int nf = kFactorial[d];
            for (int k = threadIdx.x; k < nf; k += blockDim.x) sm[k] = 0u;
            __syncthreads();
            for (int64_t i = threadIdx.x; i < npat; i += blockDim.x) {
                float v[7];
                for (int j = 0; j < d; ++j) v[j] = x[i + static_cast<int64_t>(j) * tau];
                int id = 0;
                for (int j = 0; j < d; ++j) {
                    int pos = 0;
                    for (int l = 0; l < d; ++l) pos += (v[l] < v[j] || (v[l] == v[j] && l < j)) ? 1 : 0;
                    id += j * kFactorial[d - 1 - pos];
                }
                atomicAdd(&sm[id], 1u);
            }
            __syncthreads();
            double h = 0.0;
            for (int k = threadIdx.x; k < nf; k += blockDim.x)
                if (sm[k] > 0u) {
                    const double p = static_cast<double>(sm[k]) / static_cast<double>(npat);
                    h -= p * log(p);
                }
            h = block_sum_d(h, red);
            result = nf > 1 ? h / log(static_cast<double>(nf)) : h;
        }
    } else {
        const int bins = static_cast<int>(plan.param[m]);
        double lo = CUDART_INF, hi = -CUDART_INF;
        for (int i = threadIdx.x; i < nwin; i += blockDim.x) {
            lo = fmin(lo, static_cast<double>(x[i]));
            hi = fmax(hi, static_cast<double>(x[i]));
        }
        lo = -block_max_d(-lo, red);
        hi = block_max_d(hi, red);
        const double range = (hi - lo) + 1e-10;
        unsigned char* sym = reinterpret_cast<unsigned char*>(sm);
        unsigned* keys = sm + (nwin + 15) / 16 * 4;
        unsigned* vals = keys + table_size;
        for (int i = threadIdx.x; i < nwin; i += blockDim.x) {
            const long long b = static_cast<long long>((static_cast<double>(x[i]) - lo) / range * bins);
            sym[i] = static_cast<unsigned char>(b < 0 ? 0 : (b > bins - 1 ? bins - 1 : b));
        }
        for (int q = threadIdx.x; q < table_size; q += blockDim.x) keys[q] = 0xffffffffu;
        __syncthreads();
        if (threadIdx.x == 0) {
            const unsigned mask = static_cast<unsigned>(table_size - 1);
            int shift = 32;
            for (int t = table_size; t > 1; t >>= 1) --shift;
            unsigned nodes = 1u;
            int complexity = 0;
            int64_t i = 0;
            while (i < nwin) {
                unsigned node = 0u;
                int64_t len = 1;
                while (i + len <= nwin) {
                    const unsigned key = node * 256u + sym[i + len - 1];
                    unsigned h = (key * 2654435761u) >> shift;
                    while (keys[h] != 0xffffffffu && keys[h] != key) h = (h + 1u) & mask;  // never full
                    if (keys[h] == 0xffffffffu) {
                        keys[h] = key;
                        vals[h] = nodes++;
                        ++complexity;
                        break;
                    }
                    node = vals[h];
                    ++len;
                }
                i += len;
            }
            const double nn = static_cast<double>(nwin);
            result = nwin > 1 ? complexity / (nn / (log(nn) + 1e-10)) : static_cast<double>(complexity);
        }
    }
    if (threadIdx.x == 0) out[traj * n_features + plan.col[m]] = result;
}

// Repeated values over the whole window (kinds 59..64): one block per (trajectory,
// sorted column) sorts that column's window in shared memory, as order-preserving
// keys padded to a power of two with all-ones keys (after every number), by a
// bitonic network, then counts runs of equal neighbours.  Equality is the float
// comparison, so NaN equals nothing and -0 equals +0, as in torch; the block reads
// only the first nwin sorted keys.
__global__ void __launch_bounds__(256) k_window_sorted(const float* __restrict__ win, int nwin, int pow2,
                                                       MedianPlan plan, double* __restrict__ out, int n_features)
{
    extern __shared__ uint32_t keys[];  // pow2 entries
    __shared__ double red_d[2][8];
    __shared__ unsigned red_u[3][8];
    const int64_t blk = blockIdx.x;
    const int64_t traj = blk / plan.n_sorted;
    const int m = plan.sorted_m[blk - traj * plan.n_sorted];
    const float* x = win + (traj * plan.n_med + m) * static_cast<int64_t>(nwin);
    int nan_seen = 0;
    for (int i = threadIdx.x; i < pow2; i += blockDim.x) {
        uint32_t k = 0xffffffffu;
        if (i < nwin) {
            const float v = x[i];
            nan_seen |= isnan(v) ? 1 : 0;
            k = float_key(v);
        }
        keys[i] = k;
    }
    const int any_nan = __syncthreads_or(nan_seen);
    const int half = pow2 >> 1;
    for (int k = 2; k <= pow2; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int p = threadIdx.x; p < half; p += blockDim.x) {
                const int i = ((p & ~(j - 1)) << 1) | (p & (j - 1));  // bit j of i clear
                const int l = i | j;
                const uint32_t a = keys[i], c = keys[l];
                if ((a > c) == ((i & k) == 0)) {
                    keys[i] = c;
                    keys[l] = a;
                }
            }
            __syncthreads();
        }
    }
    unsigned dups = 0, in_runs = 0, starts = 0;
    double s_runs = 0.0, s_starts = 0.0;
    for (int i = threadIdx.x; i < nwin; i += blockDim.x) {
        const float v = key_float(keys[i]);
        const bool eq_prev = i > 0 && key_float(keys[i - 1]) == v;
        const bool eq_next = i + 1 < nwin && key_float(keys[i + 1]) == v;
        dups += eq_prev ? 1u : 0u;
        if (eq_prev || eq_next) {
            ++in_runs;
            s_runs += static_cast<double>(v);
        }
        if (eq_next && !eq_prev) {
            ++starts;
            s_starts += static_cast<double>(v);
        }
    }
    for (int off = 16; off > 0; off >>= 1) {
        dups += __shfl_xor_sync(0xffffffffu, dups, off);
        in_runs += __shfl_xor_sync(0xffffffffu, in_runs, off);
        starts += __shfl_xor_sync(0xffffffffu, starts, off);
        s_runs += __shfl_xor_sync(0xffffffffu, s_runs, off);
        s_starts += __shfl_xor_sync(0xffffffffu, s_starts, off);
    }
    const int warp = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        red_u[0][warp] = dups;
        red_u[1][warp] = in_runs;
        red_u[2][warp] = starts;
        red_d[0][warp] = s_runs;
        red_d[1][warp] = s_starts;
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    const int nw = static_cast<int>(blockDim.x >> 5);
    double d = 0.0, r = 0.0, st = 0.0, sr = 0.0, ss = 0.0;
    for (int w = 0; w < nw; ++w) {
        d += red_u[0][w];
        r += red_u[1][w];
        st += red_u[2][w];
        sr += red_d[0][w];
        ss += red_d[1][w];
    }
    const double n = static_cast<double>(nwin);
    double result;
    switch (plan.kind[m]) {
        case PB_FEAT_HAS_DUPLICATE: result = d > 0.0 ? 1.0 : 0.0; break;
        case PB_FEAT_PCT_REOCCURRING_POINTS: result = st / ((n - d) + 1e-10); break;  // repeated values / distinct
        case PB_FEAT_PCT_REOCCURRING_VALUES: result = nwin <= 1 ? 0.0 : r / n; break;   // samples in runs / N
        // the reference sums sorted values times a 0/1 mask: a NaN anywhere gives NaN
        case PB_FEAT_SUM_REOCCURRING_POINTS: result = any_nan ? CUDART_NAN : sr; break;
        case PB_FEAT_SUM_REOCCURRING_VALUES: result = any_nan ? CUDART_NAN : ss; break;
        default: result = (n - d) / n; break;  // PB_FEAT_RATIO_UNIQUE_VALUES
    }
    out[traj * n_features + plan.col[m]] = result;
}

// ---------------------------------------------------------------------------
// 1-NN labelling + per-group counts.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double impute_extreme(double v)
{
    if (isnan(v)) return 1e10;
    if (isinf(v)) return v > 0 ? 1e10 : -1e10;
    return v;
}

__global__ void __launch_bounds__(256) k_label_nearest(const double* __restrict__ feat, int64_t n, int nf,
                                                       const double* __restrict__ tpl, int nt,
                                                       const int32_t* __restrict__ tpl_label, int n_classes,
                                                       const int32_t* __restrict__ status,
                                                       const int32_t* __restrict__ group_of, int n_groups,
                                                       int32_t* __restrict__ labels,
                                                       unsigned long long* __restrict__ counts)
{
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int cls;
    if (status && status[i] == PB_TRAJ_UNBOUNDED) {
        cls = n_classes;
    } else {
        double best = CUDART_INF;
        int arg = 0;
        for (int t = 0; t < nt; ++t) {
            double d2 = 0.0;
            for (int f = 0; f < nf; ++f) {
                const double d = impute_extreme(feat[i * nf + f]) - impute_extreme(__ldg(tpl + t * nf + f));
                d2 += d * d;
            }
            if (d2 < best) {  // first minimum wins on ties
                best = d2;
                arg = t;
            }
        }
        cls = __ldg(tpl_label + arg);
    }
    labels[i] = cls;
    const int g = group_of ? group_of[i] : 0;
    if (g >= 0 && g < n_groups && cls >= 0 && cls <= n_classes) atomicAdd(counts + static_cast<int64_t>(g) * (n_classes + 1) + cls, 1ull);
}

// ---------------------------------------------------------------------------
// FMA-pipe throughput probe (roofline denominator for the integrator kernels)
// ---------------------------------------------------------------------------
template <class T>
__global__ void __launch_bounds__(256) k_probe_fma(int iters, float* __restrict__ sink)
{
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    T a[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) a[j] = static_cast<T>(tid * 1e-7 + j * 1e-3);
    const T m = static_cast<T>(0.9999999), c = static_cast<T>(1e-7);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int j = 0; j < 8; ++j) a[j] = fma(a[j], m, c);
    }
    T acc = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) acc += a[j];
    sink[tid] = static_cast<float>(acc);
}

// ---------------------------------------------------------------------------
// kernel selection
// ---------------------------------------------------------------------------
template <class F>
static KFn rt_fn(F* f)
{
    KFn k;
    k.rt = reinterpret_cast<const void*>(f);
    return k;
}

template <class Sys, class R>
KernelSel select_prec()
{
    KernelSel k;
    k.smem_per_thread = Stats<Sys::S>::kBytesPerThread;
    k.plain = rt_fn(k_solve_plain<Sys, R, false>);
    k.plain_defer = rt_fn(k_solve_plain<Sys, R, true>);
    k.queue = rt_fn(k_solve_queue<Sys, R, false>);
    k.queue_defer = rt_fn(k_solve_queue<Sys, R, true>);
    k.queue_probe = rt_fn(k_solve_queue<Sys, R, true, 1>);
    k.queue_main = rt_fn(k_solve_queue<Sys, R, true, 2>);
    k.queue_main_s1 = rt_fn(k_solve_queue<Sys, R, true, 2, SampleDrain<R, 1>>);
    k.queue_main_s2 = rt_fn(k_solve_queue<Sys, R, true, 2, SampleDrain<R, 2>>);
    return k;
}

template <class Sys>
KernelSel select_kernel(int precision)
{
    return precision == PB_PREC_FP64 ? select_prec<Sys, double>() : select_prec<Sys, float>();
}

static KernelSel find_kernel(int system, int dim, int precision, int schedule)
{
    if (precision != PB_PREC_FP64 && precision != PB_PREC_MIXED) return {};
    if (schedule != PB_SCHED_PLAIN && schedule != PB_SCHED_QUEUE && schedule != PB_SCHED_PROBED) return {};
    switch (system) {
        case PB_SYS_LINEAR:
            switch (dim) {
                case 1: return select_kernel<SysLinear<1>>(precision);
                case 2: return select_kernel<SysLinear<2>>(precision);
                case 3: return select_kernel<SysLinear<3>>(precision);
                case 4: return select_kernel<SysLinear<4>>(precision);
                default: return {};
            }
        case PB_SYS_PENDULUM: return dim == 2 ? select_kernel<SysPendulum>(precision) : KernelSel{};
        case PB_SYS_DUFFING: return dim == 2 ? select_kernel<SysDuffing>(precision) : KernelSel{};
        case PB_SYS_LORENZ: return dim == 3 ? select_kernel<SysLorenz<false>>(precision) : KernelSel{};
        case PB_SYS_LORENZ_MASKED: return dim == 3 ? select_kernel<SysLorenz<true>>(precision) : KernelSel{};
        case PB_SYS_FRICTION: return dim == 2 ? select_kernel<SysFriction>(precision) : KernelSel{};
        default: return {};
    }
}

// Sampling pass for `ns` feature states (shared by every system)
template <class R, int NS>
static KFn sample_of(bool cross)
{
    return cross ? rt_fn(k_sample<R, NS, PB_MAX_CROSSING>) : rt_fn(k_sample<R, NS, 0>);
}

template <class R>
static KFn sample_kernel_r(int ns, bool cross)
{
    switch (ns) {
        case 1: return sample_of<R, 1>(cross);
        case 2: return sample_of<R, 2>(cross);
        case 3: return sample_of<R, 3>(cross);
        case 4: return sample_of<R, 4>(cross);
        case 5: return sample_of<R, 5>(cross);
        case 6: return sample_of<R, 6>(cross);
        case 7: return sample_of<R, 7>(cross);
        case 8: return sample_of<R, 8>(cross);
        default: return KFn{};
    }
}

static KFn sample_kernel(int precision, int ns, bool cross)
{
    return precision == PB_PREC_FP64 ? sample_kernel_r<double>(ns, cross) : sample_kernel_r<float>(ns, cross);
}

// launches of a kernel handle: (pb_solve_args) or (pb_solve_args, int) arguments
static cudaError_t launch_fn(const KFn& f, int64_t grid, int block, int smem, cudaStream_t st,
                             const pb_solve_args& a, const int* extra)
{
    if (grid <= 0 || grid > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
    pb_solve_args copy = a;
    int x = extra ? *extra : 0;
    void* argv[2] = {&copy, &x};
    if (f.rt) return cudaLaunchKernel(f.rt, dim3(static_cast<unsigned>(grid)), dim3(block), argv, smem, st);
    if (f.drv) return drv_launch(f.drv, static_cast<unsigned>(grid), block, smem, st, argv);
    return cudaErrorInvalidDeviceFunction;
}

// Dynamic shared memory above the 48 KB default needs an opt-in per kernel.
static cudaError_t prepare_smem(const KFn& f, int bytes)
{
    if (bytes <= 48 * 1024) return cudaSuccess;
    if (f.rt) return cudaFuncSetAttribute(f.rt, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    return drv_set_max_smem(f.drv, bytes);
}

static cudaError_t occupancy(const KFn& f, int block, int smem, int* bps)
{
    if (f.rt) return cudaOccupancyMaxActiveBlocksPerMultiprocessor(bps, f.rt, block, smem);
    return drv_occupancy(f.drv, block, smem, bps);
}

// Persistent grid for a queue kernel: resident blocks on every SM, capped by the work.
static cudaError_t persistent_grid(const KFn& f, int block, int smem, int64_t n_traj, int requested, int64_t* grid)
{
    if (requested > 0) {
        *grid = requested;
    } else {
        int dev = 0, sms = 0, bps = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e == cudaSuccess) e = occupancy(f, block, smem, &bps);
        if (e != cudaSuccess) return e;
        *grid = static_cast<int64_t>(sms) * (bps > 0 ? bps : 1);
    }
    const int64_t need = (n_traj + block - 1) / block;
    if (*grid > need) *grid = need;
    return cudaSuccess;
}

// Radix-sort temporary storage for the probed schedule's longest-first order.
static size_t sort_temp_bytes(int64_t n)
{
    size_t bytes = 0;
    if (cub::DeviceRadixSort::SortPairsDescending(nullptr, bytes, static_cast<const unsigned*>(nullptr),
                                                  static_cast<unsigned*>(nullptr),
                                                  static_cast<const unsigned*>(nullptr),
                                                  static_cast<unsigned*>(nullptr), static_cast<int>(n)) !=
        cudaSuccess)
        return 0;
    return bytes;
}

// Stable descending sort of the probe-phase step counts: the main phase then
// takes the longest predicted trajectories first, so they start on every SM in
// the first wave and the short ones fill in at the end.
static cudaError_t sort_by_probe(const pb_solve_args& a, const ScratchLayout& sl, cudaStream_t st)
{
    unsigned char* base = static_cast<unsigned char*>(a.scratch);
    size_t bytes = sort_temp_bytes(a.n_traj);
    if (bytes == 0) return cudaErrorInvalidValue;
    int end_bit = 1;
    while (end_bit < 32 && (static_cast<int64_t>(1) << end_bit) <= a.max_steps) ++end_bit;
    return cub::DeviceRadixSort::SortPairsDescending(
        base + sl.sort_tmp_off, bytes, reinterpret_cast<const unsigned*>(base + sl.key_in_off),
        reinterpret_cast<unsigned*>(base + sl.key_out_off), reinterpret_cast<const unsigned*>(base + sl.val_in_off),
        reinterpret_cast<unsigned*>(base + sl.val_out_off), static_cast<int>(a.n_traj), 0, end_bit, st);
}

static int count_median_cols(const pb_solve_args& a, MedianPlan* plan)
{
    int m = 0, np = 0, ns = 0, nsp = 0, nsy = 0;
    for (int c = 0; c < a.n_features; ++c)
        if (PB_FEAT_IS_WINDOW(a.feat_kind[c])) {
            if (plan) {
                plan->col[m] = c;
                plan->kind[m] = a.feat_kind[c];
                plan->param[m] = a.feat_param[c];
                plan->param2[m] = a.feat_param2[c];
                plan->peak_idx[m] = a.feat_kind[c] == PB_FEAT_NUMBER_PEAKS ? np : -1;
            }
            np += a.feat_kind[c] == PB_FEAT_NUMBER_PEAKS;
            if (plan && PB_FEAT_IS_SORTED(a.feat_kind[c])) plan->sorted_m[ns] = m;
            ns += PB_FEAT_IS_SORTED(a.feat_kind[c]) ? 1 : 0;
            if (plan && PB_FEAT_IS_SPECTRAL(a.feat_kind[c])) plan->spectral_m[nsp] = m;
            nsp += PB_FEAT_IS_SPECTRAL(a.feat_kind[c]) ? 1 : 0;
            if (plan && PB_FEAT_IS_SYMBOLIC(a.feat_kind[c])) plan->symbolic_m[nsy] = m;
            nsy += PB_FEAT_IS_SYMBOLIC(a.feat_kind[c]) ? 1 : 0;
            ++m;
        }
    if (plan) {
        plan->n_sorted = ns;
        plan->n_spectral = nsp;
        plan->n_symbolic = nsy;
        plan->n_med = m;
        plan->n_peak_cols = np;
        plan->peak_cap = a.peak_cap;
        plan->peaks_out = a.peak_cap > 0 ? a.peaks_out : nullptr;
    }
    return m;
}

static int map_cuda(cudaError_t e)
{
    if (e == cudaSuccess) return PB_SUCCESS;
    if (e == cudaErrorMemoryAllocation) return PB_EALLOC;
    if (e == cudaErrorLaunchFailure || e == cudaErrorLaunchOutOfResources || e == cudaErrorInvalidConfiguration)
        return PB_ESOLVE;
    return PB_ECUDA;
}

int validate_args(const pb_solve_args* a, bool user_system)
{
    if (!a) return PB_EINVAL;
    if ((a->system == PB_SYS_USER) != user_system) return PB_EINVALID_ODE;
    if (a->n_traj < 0 || a->n_ic < 0 || a->dim <= 0) return PB_EINVAL;
    if (a->n_traj > 0 && (!a->y0 || !a->params || !a->save_ts)) return PB_EINVAL;
    if (a->n_params < 0 || a->n_params > PB_MAX_PARAMS) return PB_EINVAL;
    if (a->n_save < 1 || a->win_begin < 0 || a->win_begin >= a->n_save) return PB_EINVAL;
    if (a->n_features < 0 || a->n_features > PB_MAX_FEATURES) return PB_EINVAL;
    if (a->y0_dtype != PB_DTYPE_F32 && a->y0_dtype != PB_DTYPE_F64) return PB_EINVAL;
    if (a->y_out_dtype != PB_DTYPE_F32 && a->y_out_dtype != PB_DTYPE_F64) return PB_EINVAL;
    if (!(a->rtol >= 0.0) || !(a->atol >= 0.0) || !(a->rtol + a->atol > 0.0)) return PB_EINVAL;
    if (!(a->t1 >= a->t0) || a->max_steps < 0) return PB_EINVAL;
    int n_cross = 0;
    for (int c = 0; c < a->n_features; ++c) {
        if (a->feat_state[c] < 0 || a->feat_state[c] >= a->dim) return PB_EINVAL;
        const int kind = a->feat_kind[c];
        const double prm = a->feat_param[c];
        if (kind < PB_FEAT_MEDIAN || kind > PB_FEAT_LAST_KIND) return PB_EINVAL;
        if (kind == PB_FEAT_QUANTILE && !(prm >= 0.0 && prm <= 1.0)) return PB_EINVAL;
        const bool int_param = kind == PB_FEAT_NUMBER_PEAKS || kind == PB_FEAT_AUTOCORRELATION ||
                               (kind >= PB_FEAT_FFT_REAL && kind <= PB_FEAT_FFT_ANGLE) || kind == PB_FEAT_C3 ||
                               kind == PB_FEAT_TIME_REVERSAL || kind == PB_FEAT_SPKT_WELCH;
        if (int_param && !(prm >= 0.0 && prm <= 1e6 && prm == static_cast<double>(static_cast<int>(prm))))
            return PB_EINVAL;
        if (kind == PB_FEAT_CID_CE && !(prm == 0.0 || prm == 1.0)) return PB_EINVAL;
        if (kind == PB_FEAT_INDEX_MASS_QUANTILE && !(prm >= 0.0 && prm <= 1.0)) return PB_EINVAL;
        if (kind == PB_FEAT_BINNED_ENTROPY && !(prm >= 1.0 && prm <= 256.0 && prm == static_cast<double>(static_cast<int>(prm))))
            return PB_EINVAL;
        if (kind == PB_FEAT_MEAN_N_ABS_MAX && !(prm >= 1.0 && prm <= 64.0 && prm == static_cast<double>(static_cast<int>(prm))))
            return PB_EINVAL;
        if (PB_FEAT_IS_SORTED(kind) && a->n_save - a->win_begin > PB_SORTED_WINDOW_MAX) return PB_EUNSUPPORTED;
        if (PB_FEAT_IS_SPECTRAL(kind) && a->n_save - a->win_begin > PB_SPECTRAL_WINDOW_MAX) return PB_EUNSUPPORTED;
        if (kind == PB_FEAT_LEMPEL_ZIV && a->n_save - a->win_begin > PB_SYMBOLIC_WINDOW_MAX) return PB_EUNSUPPORTED;
        const double prm2 = a->feat_param2[c];
        const auto is_int = [](double v, double lo, double hi) {
            return v >= lo && v <= hi && v == static_cast<double>(static_cast<int>(v));
        };
        if (kind == PB_FEAT_PARTIAL_AUTOCORRELATION && !is_int(prm, 0.0, 63.0)) return PB_EINVAL;
        if (kind == PB_FEAT_PERMUTATION_ENTROPY && !(is_int(prm, 1.0, 1e6) && is_int(prm2, 1.0, 7.0))) return PB_EINVAL;
        if (kind == PB_FEAT_LEMPEL_ZIV && !is_int(prm, 1.0, 255.0)) return PB_EINVAL;
        if (kind >= PB_FEAT_AGG_TREND_MEAN && kind <= PB_FEAT_AGG_TREND_MAX &&
            !(is_int(prm, 1.0, 1e9) && is_int(prm2, 0.0, 4.0)))
            return PB_EINVAL;
        if (kind == PB_FEAT_AR_COEFFICIENT && !(is_int(prm, 1.0, 10.0) && is_int(prm2, 0.0, 1e6))) return PB_EINVAL;
        if (kind == PB_FEAT_CWT && !(is_int(prm, 1.0, 1e4) && is_int(prm2, -1.0, 1e9))) return PB_EINVAL;
        if (kind == PB_FEAT_NUMBER_CWT_PEAKS && !is_int(prm, 0.0, 64.0)) return PB_EINVAL;
        if (kind == PB_FEAT_LYAP_R) {
            const int e = static_cast<int>(prm) / 1024, tl = static_cast<int>(prm) % 1024;
            if (!(is_int(prm, 1024.0, 64.0 * 1024.0 + 1023.0) && e >= 1 && tl >= 1 && is_int(prm2, 1.0, 100000.0)))
                return PB_EINVAL;
            if (a->n_save - a->win_begin > PB_SPECTRAL_WINDOW_MAX) return PB_EUNSUPPORTED;
        }
        if (kind == PB_FEAT_CORR_DIM) {
            if (!(is_int(prm, 1.0, 16.0) && is_int(prm2, 1024.0, 1024.0 * 100000.0 + 1023.0))) return PB_EINVAL;
            if (static_cast<int>(prm2) % 1024 < 1) return PB_EINVAL;
            if (a->n_save - a->win_begin > PB_SPECTRAL_WINDOW_MAX) return PB_EUNSUPPORTED;
        }
        if ((kind == PB_FEAT_FRIEDRICH || kind == PB_FEAT_LANGEVIN) && !(is_int(prm, 0.0, 6.0) && is_int(prm2, 0.0, 1e6)))
            return PB_EINVAL;
        if ((kind == PB_FEAT_ACF_PERIOD_STRENGTH || kind == PB_FEAT_ACF_PERIOD_LAG) && !is_int(prm, 0.0, 1e9))
            return PB_EINVAL;
        if (kind >= PB_FEAT_AGG_AUTOCORR_MEAN && kind <= PB_FEAT_AGG_AUTOCORR_VAR && !is_int(prm, 0.0, 128.0))
            return PB_EINVAL;
        if (kind == PB_FEAT_ENERGY_RATIO_BY_CHUNKS && !(is_int(prm, 1.0, 1e6) && is_int(prm2, 0.0, 1e6)))
            return PB_EINVAL;
        if (kind >= PB_FEAT_CHANGE_QUANTILES_MEAN && kind <= PB_FEAT_CHANGE_QUANTILES_ABS_VAR &&
            !(prm >= 0.0 && prm <= 1.0 && prm2 >= 0.0 && prm2 <= 1.0))
            return PB_EINVAL;
        if ((a->feat_kind[c] == PB_FEAT_SYNC_DEV) != (a->system == PB_SYS_ROSSLER_NET)) return PB_EUNSUPPORTED;
        n_cross += a->feat_kind[c] == PB_FEAT_CROSSINGS;
    }
    if (n_cross > PB_MAX_CROSSING) return PB_EUNSUPPORTED;
    if (a->n_features > 0 && !a->features_out) return PB_EINVAL;
    if (a->dense_mode != PB_DENSE_INLINE && a->dense_mode != PB_DENSE_DEFERRED) return PB_EINVAL;
    if (a->window_record_cap < 0) return PB_EINVAL;
    if (a->peak_cap < 0 || (a->peaks_out && a->peak_cap == 0)) return PB_EINVAL;
    for (int c = 0; c < a->n_features; ++c)
        if (a->feat_state[c] >= PB_MAX_STAT_STATES) return PB_EUNSUPPORTED;
    switch (a->layout) {
        case PB_LAYOUT_SINGLE:
            if (a->n_ic < a->n_traj || a->n_param_rows < 1) return PB_EINVAL;
            break;
        case PB_LAYOUT_CROSS:
            if (a->n_param_rows < 1 || a->n_ic * a->n_param_rows != a->n_traj) return PB_EINVAL;
            break;
        case PB_LAYOUT_INDEXED:
            if (!a->param_index && a->n_traj > 0) return PB_EINVAL;
            if (a->n_ic < a->n_traj || a->n_param_rows < 1) return PB_EINVAL;
            break;
        default: return PB_EINVAL;
    }
    if ((a->schedule == PB_SCHED_QUEUE || a->schedule == PB_SCHED_PROBED) && !a->queue_counter) return PB_EINVAL;
    if (a->schedule == PB_SCHED_PROBED && a->n_traj > 0x7fffffffLL) return PB_EINVAL;  // 32-bit sort values
    if (a->block_size < 0 || (a->block_size % 32) != 0 || a->block_size > 256) return PB_EINVAL;
    if (a->refill_lanes < 0 || a->refill_lanes > 32) return PB_EINVAL;
    return PB_SUCCESS;
}

// The passes of one solve: pass 1 (plain, queue or probe + sort + main), the
// sampling pass and the redo of record overflows for deferred dense output, then
// the median pass.  `a` has been validated.
int solve_with(const KernelSel& k, const pb_solve_args& a, cudaStream_t st)
{
    const int zero = 0, one = 1;
    if (a.n_traj == 0) return PB_SUCCESS;
    const ScratchLayout sl = scratch_layout(a);
    if (sl.total > 0 && !a.scratch) return PB_EINVAL;
    if (sl.deferred && !a.queue_counter) return PB_EINVAL;  // the redo pass runs on the queue
    // defaults from the launch-shape sweep: 64 for the queue schedules, 128 plain
    const int block = a.block_size > 0 ? a.block_size : (a.schedule == PB_SCHED_PLAIN ? 128 : 64);
    const int smem = k.smem_per_thread * block;
    cudaError_t e = cudaSuccess;
    const int64_t plain_grid = (a.n_traj + block - 1) / block;
    if (plain_grid > 0x7fffffffLL) return PB_EINVAL;

    if (sl.deferred) {
        bool any_cross = false;
        for (int c = 0; c < a.n_features; ++c) any_cross |= a.feat_kind[c] == PB_FEAT_CROSSINGS;
        const int ns = count_stat_states(a);
        if (a.precision != PB_PREC_FP64) {  // FP32 offsets of the save grid, for the sampling
            k_split_saves<<<(a.n_save + 255) / 256, 256, 0, st>>>(
                a.save_ts, a.n_save,
                reinterpret_cast<float2*>(static_cast<unsigned char*>(a.scratch) + sl.split_off));
            e = cudaGetLastError();
            if (e != cudaSuccess) return map_cuda(e);
        }
        // pass 1: integrate, one record per window step holding save points
        if (sl.probed) {
            // probe phase, longest-first sort of its step counts, main phase
            int64_t grid = 0;
            e = persistent_grid(k.queue_probe, block, 0, a.n_traj, a.grid_blocks, &grid);
            if (e == cudaSuccess) e = cudaMemsetAsync(a.queue_counter, 0, sizeof(unsigned long long), st);
            if (e != cudaSuccess) return map_cuda(e);
            e = launch_fn(k.queue_probe, grid, block, 0, st, a, &zero);
            if (e == cudaSuccess) e = sort_by_probe(a, sl, st);
            // main phase, with the sampling drained into it where a variant exists
            // (1 or 2 feature states, no crossing counts); the pass below samples
            // whatever it leaves
            KFn main = k.queue_main;
            if (!any_cross && ns == 1 && k.queue_main_s1.ok()) main = k.queue_main_s1;
            if (!any_cross && ns == 2 && k.queue_main_s2.ok()) main = k.queue_main_s2;
            if (e == cudaSuccess) e = persistent_grid(main, block, 0, a.n_traj, a.grid_blocks, &grid);
            if (e == cudaSuccess) e = cudaMemsetAsync(a.queue_counter, 0, sizeof(unsigned long long), st);
            if (e == cudaSuccess)
                e = cudaMemsetAsync(static_cast<unsigned char*>(a.scratch) + sl.drain_off, 0,
                                    static_cast<size_t>(drain_bytes(sl, a.n_traj)), st);
            if (e != cudaSuccess) return map_cuda(e);
            e = launch_fn(main, grid, block, 0, st, a, &zero);
        } else if (a.schedule != PB_SCHED_PLAIN) {
            int64_t grid = 0;
            e = persistent_grid(k.queue_defer, block, 0, a.n_traj, a.grid_blocks, &grid);
            if (e == cudaSuccess) e = cudaMemsetAsync(a.queue_counter, 0, sizeof(unsigned long long), st);
            if (e != cudaSuccess) return map_cuda(e);
            e = launch_fn(k.queue_defer, grid, block, 0, st, a, &zero);
        } else {
            e = launch_fn(k.plain_defer, plain_grid, block, 0, st, a, nullptr);
        }
        if (e != cudaSuccess) return map_cuda(e);
        // pass 2: one warp per trajectory evaluates its save points and reduces the statistics
        const int64_t sblocks = (a.n_traj + 3) / 4;
        if (sblocks > 0x7fffffffLL) return PB_EINVAL;
        const KFn sample = sample_kernel(a.precision, ns, any_cross);
        if (!sample.ok()) return PB_EUNSUPPORTED;
        e = launch_fn(sample, sblocks, 128, 0, st, a, nullptr);
        if (e != cudaSuccess) return map_cuda(e);
        // pass 3: trajectories that exceeded the record capacity, inline
        int64_t grid = 0;
        e = prepare_smem(k.queue, smem);
        if (e == cudaSuccess) e = persistent_grid(k.queue, block, smem, a.n_traj, a.grid_blocks, &grid);
        if (e == cudaSuccess) e = cudaMemsetAsync(a.queue_counter, 0, sizeof(unsigned long long), st);
        if (e != cudaSuccess) return map_cuda(e);
        e = launch_fn(k.queue, grid, block, smem, st, a, &one);
    } else if (a.schedule != PB_SCHED_PLAIN) {
        int64_t grid = 0;
        e = prepare_smem(k.queue, smem);
        if (e == cudaSuccess) e = persistent_grid(k.queue, block, smem, a.n_traj, a.grid_blocks, &grid);
        if (e == cudaSuccess) e = cudaMemsetAsync(a.queue_counter, 0, sizeof(unsigned long long), st);
        if (e != cudaSuccess) return map_cuda(e);
        e = launch_fn(k.queue, grid, block, smem, st, a, &zero);
    } else {
        e = prepare_smem(k.plain, smem);
        if (e != cudaSuccess) return map_cuda(e);
        e = launch_fn(k.plain, plain_grid, block, smem, st, a, nullptr);
    }
    if (e != cudaSuccess) return map_cuda(e);
    MedianPlan plan;
    if (count_median_cols(a, &plan) > 0) {
        const int64_t rows = a.n_traj * plan.n_med;
        const int64_t blocks = (rows + 7) / 8;
        if (blocks > 0x7fffffffLL) return PB_EINVAL;
        k_window<<<static_cast<unsigned>(blocks), 256, 0, st>>>(
            reinterpret_cast<const float*>(static_cast<const unsigned char*>(a.scratch) + sl.median_off), a.n_traj,
            a.n_save - a.win_begin, plan, a.features_out, a.n_features);
        e = cudaGetLastError();
        if (e != cudaSuccess) return map_cuda(e);
        if (plan.n_sorted > 0) {
            const int nwin = a.n_save - a.win_begin;  // <= PB_SORTED_WINDOW_MAX (validated)
            int pow2 = 1;
            while (pow2 < nwin) pow2 <<= 1;
            const int64_t sblocks = a.n_traj * plan.n_sorted;
            if (sblocks > 0x7fffffffLL) return PB_EINVAL;
            const size_t smem = static_cast<size_t>(pow2) * sizeof(uint32_t);
            if (smem > 48 * 1024)
                e = cudaFuncSetAttribute(k_window_sorted, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
            if (e != cudaSuccess) return map_cuda(e);
            k_window_sorted<<<static_cast<unsigned>(sblocks), 256, smem, st>>>(
                reinterpret_cast<const float*>(static_cast<const unsigned char*>(a.scratch) + sl.median_off), nwin,
                pow2, plan, a.features_out, a.n_features);
            e = cudaGetLastError();
            if (e != cudaSuccess) return map_cuda(e);
        }
        if (plan.n_spectral > 0) {
            const int nwin = a.n_save - a.win_begin;  // <= PB_SPECTRAL_WINDOW_MAX (validated)
            const int64_t sblocks = a.n_traj * plan.n_spectral;
            if (sblocks > 0x7fffffffLL) return PB_EINVAL;
            const size_t smem = static_cast<size_t>(nwin / 2 + 1) * sizeof(double);
            if (smem > 48 * 1024)
                e = cudaFuncSetAttribute(k_window_spectrum, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
            if (e != cudaSuccess) return map_cuda(e);
            k_window_spectrum<<<static_cast<unsigned>(sblocks), 256, smem, st>>>(
                reinterpret_cast<const float*>(static_cast<const unsigned char*>(a.scratch) + sl.median_off), nwin,
                plan, a.features_out, a.n_features);
            e = cudaGetLastError();
            if (e != cudaSuccess) return map_cuda(e);
        }
        if (plan.n_symbolic > 0) {
            const int nwin = a.n_save - a.win_begin;
            bool lz = false;
            size_t cd = 0;  // correlation_dimension: window floats, radii (doubles), a histogram per warp
            for (int q = 0; q < plan.n_symbolic; ++q) {
                const int mq = plan.symbolic_m[q];
                lz |= plan.kind[mq] == PB_FEAT_LEMPEL_ZIV;
                if (plan.kind[mq] == PB_FEAT_LYAP_R)  // window floats and a neighbour index per vector
                    cd = std::max(cd, static_cast<size_t>((nwin + 3) / 4 * 16) + sizeof(int) * nwin);
                if (plan.kind[mq] == PB_FEAT_CORR_DIM) {
                    const size_t nr = static_cast<size_t>(static_cast<int>(plan.param2[mq]) % 1024);
                    cd = std::max(cd, static_cast<size_t>((nwin + 3) / 4 * 16) + nr * sizeof(double) +
                                          8 * nr * sizeof(unsigned));
                }
            }
            // trie table: a power of two >= 2 (nwin + 1) entries (at most half full), keys and children
            int table = 1;
            while (table < 2 * (nwin + 1)) table <<= 1;
            size_t smem = 5040 * sizeof(unsigned);  // the permutation histogram (d <= 7)
            if (lz) smem = std::max(smem, static_cast<size_t>((nwin + 15) / 16 * 16) + 2 * sizeof(unsigned) * table);
            smem = std::max(smem, cd);
            const int64_t sblocks = a.n_traj * plan.n_symbolic;
            if (sblocks > 0x7fffffffLL) return PB_EINVAL;
            if (smem > 48 * 1024)
                e = cudaFuncSetAttribute(k_window_symbolic, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
            if (e != cudaSuccess) return map_cuda(e);
            k_window_symbolic<<<static_cast<unsigned>(sblocks), 256, smem, st>>>(
                reinterpret_cast<const float*>(static_cast<const unsigned char*>(a.scratch) + sl.median_off), nwin,
                table, plan, a.features_out, a.n_features);
            e = cudaGetLastError();
            if (e != cudaSuccess) return map_cuda(e);
        }
    }
    return PB_SUCCESS;
}

}  // namespace pb

using namespace pb;

extern "C" {

// 101: pb_solve_args gained feat_param2; 102: refill_lanes (in place of a padding word)
int32_t pb_abi_version(void) { return 102; }

const char* pb_error_string(int32_t s)
{
    switch (s) {
        case PB_SUCCESS: return "success";
        case PB_EINVALID_ODE: return "invalid ODE: unknown system id / dimension";
        case PB_EALLOC: return "device memory allocation failed";
        case PB_ESOLVE: return "solver kernel failed to launch or run";
        case PB_EINVAL: return "invalid argument";
        case PB_ECUDA: return "CUDA runtime error";
        case PB_EUNSUPPORTED: return "unsupported request";
        case PB_ECOMPILE: return "runtime compilation of the right-hand side failed";
        case PB_ESCRATCH_LIMIT: return "request exceeds the fixed scratch of the allocation-free entry point";
        default: return "unknown error";
    }
}

int64_t pb_solve_scratch_bytes(const pb_solve_args* a)
{
    if (!a || a->n_traj < 0 || a->n_save < 1 || a->win_begin < 0 || a->win_begin >= a->n_save) return -1;
    // the layout walks feat_kind / feat_state up to n_features: bound it to the arrays first
    if (a->n_features < 0 || a->n_features > PB_MAX_FEATURES) return -1;
    const ScratchLayout sl = scratch_layout(*a);
    if (!sl.probed) return sl.total;
    if (a->n_traj > 0x7fffffffLL) return -1;
    const size_t tmp = sort_temp_bytes(a->n_traj);
    return tmp == 0 && a->n_traj > 0 ? -1 : align_up(sl.total + static_cast<int64_t>(tmp), 256);
}

int pb_query_occupancy(int32_t system, int32_t dim, int32_t precision, int32_t schedule, int32_t block_size,
                       int32_t* blocks_per_sm, int32_t* num_sms)
{
    KernelSel k = find_kernel(system, dim, precision, schedule);
    if (!k.plain.ok()) return PB_EINVALID_ODE;
    if (block_size <= 0 || block_size % 32 || block_size > 256) return PB_EINVAL;
    int dev = 0, bps = 0, sms = 0;
    const int smem = k.smem_per_thread * block_size;
    const KFn& f = schedule != PB_SCHED_PLAIN ? k.queue : k.plain;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = prepare_smem(f, smem);
    if (e == cudaSuccess) e = occupancy(f, block_size, smem, &bps);
    if (e != cudaSuccess) return map_cuda(e);
    if (blocks_per_sm) *blocks_per_sm = bps;
    if (num_sms) *num_sms = sms;
    return PB_SUCCESS;
}

static int solve_network(const pb_solve_args& a, cudaStream_t st)
{
    if (a.dim % 3 != 0 || a.dim / 3 < 1 || a.dim / 3 > kNetMaxNodes) return PB_EINVALID_ODE;
    if (!a.csr_row || !a.csr_col || a.n_params < 4 || !a.queue_counter) return PB_EINVAL;
    if (a.y_full_out) return PB_EUNSUPPORTED;  // features come from the final state
    if (a.n_traj == 0) return PB_SUCCESS;
    const int n_nodes = a.dim / 3;
    auto k = a.precision == PB_PREC_FP64 ? k_network<double, 4> : k_network<float, 4>;
    int dev = 0, sms = 0, bps = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k, 128, 0);
    if (e == cudaSuccess) e = cudaMemsetAsync(a.queue_counter, 0, sizeof(unsigned long long), st);
    if (e != cudaSuccess) return map_cuda(e);
    int64_t grid = static_cast<int64_t>(sms) * (bps > 0 ? bps : 1);
    const int64_t need = (a.n_traj + 3) / 4;  // 4 warps (trajectories in flight) per block
    if (grid > need) grid = need;
    k<<<static_cast<unsigned>(grid), 128, 0, st>>>(a, n_nodes);
    return map_cuda(cudaGetLastError());
}

int pb_solve_batch(const pb_solve_args* args, void* stream)
{
    int v = validate_args(args, false);
    if (v != PB_SUCCESS) return v;
    const pb_solve_args& a = *args;
    if (a.system == PB_SYS_ROSSLER_NET) return solve_network(a, static_cast<cudaStream_t>(stream));
    KernelSel k = find_kernel(a.system, a.dim, a.precision, a.schedule);
    if (!k.plain.ok()) return PB_EINVALID_ODE;
    return solve_with(k, a, static_cast<cudaStream_t>(stream));
}

int pb_probe_fma(int32_t precision, int32_t blocks, int32_t iters, float* sink, void* stream)
{
    if (blocks <= 0 || iters <= 0 || !sink) return PB_EINVAL;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (precision == PB_PREC_FP64)
        k_probe_fma<double><<<blocks, 256, 0, st>>>(iters, sink);
    else if (precision == PB_PREC_MIXED)
        k_probe_fma<float><<<blocks, 256, 0, st>>>(iters, sink);
    else
        return PB_EINVAL;
    return map_cuda(cudaGetLastError());
}

int pb_label_nearest(const double* features, int64_t n, int32_t n_features, const double* templates,
                     int32_t n_templates, const int32_t* tpl_label, int32_t n_classes, const int32_t* status,
                     const int32_t* group_of, int32_t n_groups, int32_t* labels_out, int64_t* counts_out,
                     void* stream)
{
    if (n < 0 || n_features < 0 || n_templates < 1 || n_classes < 1 || n_groups < 1) return PB_EINVAL;
    if (!templates || !tpl_label || !labels_out || !counts_out) return PB_EINVAL;
    if (n > 0 && n_features > 0 && !features) return PB_EINVAL;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemsetAsync(counts_out, 0, sizeof(int64_t) * n_groups * (n_classes + 1), st);
    if (e != cudaSuccess) return map_cuda(e);
    if (n == 0) return PB_SUCCESS;
    const int64_t blocks = (n + 255) / 256;
    if (blocks > 0x7fffffffLL) return PB_EINVAL;
    k_label_nearest<<<static_cast<unsigned>(blocks), 256, 0, st>>>(
        features, n, n_features, templates, n_templates, tpl_label, n_classes, status, group_of, n_groups,
        labels_out, reinterpret_cast<unsigned long long*>(counts_out));
    e = cudaGetLastError();
    return map_cuda(e);
}

}  // extern "C"
