// Networks of coupled oscillators: one warp integrates one trajectory.
//
// The coupled Rössler network of the reference
// (case_studies/rossler_network/rossler_network_jax_ode.py:53-79):
//   dx_i/dt = -y_i - z_i + K * sum_{j in N(i)} (x_j - x_i)
//   dy_i/dt = x_i + a y_i
//   dz_i/dt = b + z_i (x_i - c)
// with the state laid out [x_0..x_{n-1}, y_0.., z_0..] and the graph given as a
// CSR adjacency (both directions of every edge).  Lane l owns nodes l, l+32,
// l+64, l+96 (NPL = 4 nodes per lane, n <= 128); each stage publishes its x
// components to shared memory so every lane can form its nodes' Laplacian.
// The RMS error norm, the unbounded check and the synchronisation features are
// warp reductions, so step acceptance and step size are uniform across the warp
// (no divergence).  The step, control and initial step are those of
// src/zigode/src/solver/dopri5_generic.zig (see pb_dopri5.cuh).
//
// Features (PB_FEAT_SYNC_DEV, case_studies/rossler_network/
// synchronization_feature_extractor.py:73-106): at the final save point t1,
// max_i - min_i over the nodes of block feat_state (0 = x, 1 = y, 2 = z), or
// the largest of the three (feat_state = 3).
#pragma once
#include <cuda_runtime.h>
#include <math_constants.h>
#include <stdint.h>

#include <type_traits>

#include "pb_dopri5.cuh"

namespace pb {

constexpr int kNetMaxNodes = 128;
constexpr int kNetMaxEdges = 4096;  // directed entries of the CSR held in shared memory

template <class R>
struct NetShared {
    int row[kNetMaxNodes + 1];
    int col[kNetMaxEdges];
    R xs[8][kNetMaxNodes];  // per-warp exchange of x (up to 8 warps per block)
};

__device__ __forceinline__ double warp_sum(double v)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_max(double v)
{
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ double warp_min(double v)
{
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

template <class R, int NPL>
struct NetWarp {
    using V = R[3][NPL];
    int n, lane;
    R a, b, c, K;
    R* xs;
    const NetShared<R>* sh;

    __device__ __forceinline__ bool owns(int j) const { return lane + 32 * j < n; }

    // du = f(u) for this lane's nodes (collective over the warp)
    __device__ void rhs(const V& u, V& du) const
    {
#pragma unroll
        for (int j = 0; j < NPL; ++j)
            if (owns(j)) xs[lane + 32 * j] = u[0][j];
        __syncwarp();
#pragma unroll
        for (int j = 0; j < NPL; ++j) {
            if (!owns(j)) {
                du[0][j] = du[1][j] = du[2][j] = R(0);
                continue;
            }
            const int node = lane + 32 * j;
            R lap = R(0);
            for (int e = sh->row[node]; e < sh->row[node + 1]; ++e) lap += xs[sh->col[e]] - u[0][j];
            du[0][j] = -u[1][j] - u[2][j] + K * lap;
            du[1][j] = u[0][j] + a * u[1][j];
            du[2][j] = b + u[2][j] * (u[0][j] - c);
        }
        __syncwarp();
    }
};

template <class R, int NPL>
__global__ void __launch_bounds__(128) k_network(const pb_solve_args a, int n_nodes)
{
    __shared__ NetShared<R> sh;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // load the graph into shared memory, checking it: rows nondecreasing in
    // [0, n_dir], n_dir <= kNetMaxEdges, every column a node index
    const int n_dir = __ldg(a.csr_row + n_nodes);
    int bad = (n_dir < 0 || n_dir > kNetMaxEdges || __ldg(a.csr_row) != 0) ? 1 : 0;
    for (int i = threadIdx.x; i <= n_nodes; i += blockDim.x) {
        const int r = __ldg(a.csr_row + i);
        sh.row[i] = r;
        if (r < 0 || r > n_dir || (i > 0 && r < __ldg(a.csr_row + i - 1))) bad = 1;
    }
    if (!bad)
        for (int i = threadIdx.x; i < n_dir; i += blockDim.x) {
            const int cidx = __ldg(a.csr_col + i);
            sh.col[i] = cidx;
            if (cidx < 0 || cidx >= n_nodes) bad = 1;
        }
    const bool graph_ok = !__syncthreads_or(bad);
    using V = R[3][NPL];
    NetWarp<R, NPL> W;
    W.n = n_nodes;
    W.lane = lane;
    W.xs = sh.xs[warp];
    W.sh = &sh;
    const double dim = 3.0 * n_nodes;
    const bool mixed = std::is_same<R, float>::value;

    while (true) {
        unsigned long long qq = 0;
        if (lane == 0) qq = atomicAdd(a.queue_counter, 1ull);
        qq = __shfl_sync(0xffffffffu, qq, 0);
        if (static_cast<int64_t>(qq) >= a.n_traj) break;
        const int64_t q = static_cast<int64_t>(qq);
        const int64_t traj = a.order ? static_cast<int64_t>(__ldg(a.order + q)) : q;
        if (traj < 0 || traj >= a.n_traj) continue;  // an order entry out of range is ignored

        int64_t ic = traj, prow = 0;
        if (a.layout == PB_LAYOUT_CROSS) {
            ic = traj / a.n_param_rows;
            prow = traj - ic * a.n_param_rows;
        } else if (a.layout == PB_LAYOUT_INDEXED) {
            prow = __ldg(a.param_index + traj);
        }
        int status = graph_ok ? PB_TRAJ_OK : PB_TRAJ_BAD_INPUT;
        if (prow < 0 || prow >= a.n_param_rows) {
            prow = 0;
            status = PB_TRAJ_BAD_INPUT;
        }
        W.a = static_cast<R>(__ldg(a.params + prow * a.n_params + 0));
        W.b = static_cast<R>(__ldg(a.params + prow * a.n_params + 1));
        W.c = static_cast<R>(__ldg(a.params + prow * a.n_params + 2));
        W.K = static_cast<R>(__ldg(a.params + prow * a.n_params + 3));

        V y, yc, k1, k2, k3, k4, k5, k6, k7, ys, d, yn;
        double y0d[3][NPL];
#pragma unroll
        for (int blk = 0; blk < 3; ++blk)
#pragma unroll
            for (int j = 0; j < NPL; ++j) {
                const int node = lane + 32 * j;
                double v = 0.0;
                if (node < n_nodes) {
                    const int64_t idx = ic * a.dim + blk * n_nodes + node;
                    v = (a.y0_dtype == PB_DTYPE_F64) ? __ldg(static_cast<const double*>(a.y0) + idx)
                                                     : static_cast<double>(__ldg(static_cast<const float*>(a.y0) + idx));
                }
                y0d[blk][j] = v;
                y[blk][j] = static_cast<R>(v);
                yc[blk][j] = R(0);
            }
        if (!graph_ok) W.n = 0;  // a rejected graph is never read; the trajectory reports BAD_INPUT
        // initial step (dopri5_generic.zig:270-321), norms reduced over the warp
        W.rhs(y, k1);
        double s0 = 0.0, s1 = 0.0;
#pragma unroll
        for (int blk = 0; blk < 3; ++blk)
#pragma unroll
            for (int j = 0; j < NPL; ++j) {
                if (!W.owns(j)) continue;
                const double sc = a.atol + fabs(y0d[blk][j]) * a.rtol;
                const double r0 = y0d[blk][j] / sc, r1 = static_cast<double>(k1[blk][j]) / sc;
                s0 += r0 * r0;
                s1 += r1 * r1;
            }
        const double d0 = sqrt(warp_sum(s0) / dim), d1 = sqrt(warp_sum(s1) / dim);
        const double h0 = (d0 < 1e-5 || d1 < 1e-5) ? 1e-6 : 0.01 * d0 / d1;
#pragma unroll
        for (int blk = 0; blk < 3; ++blk)
#pragma unroll
            for (int j = 0; j < NPL; ++j)
                ys[blk][j] = static_cast<R>(y0d[blk][j] + h0 * static_cast<double>(k1[blk][j]));
        W.rhs(ys, k2);
        double s2 = 0.0;
#pragma unroll
        for (int blk = 0; blk < 3; ++blk)
#pragma unroll
            for (int j = 0; j < NPL; ++j) {
                if (!W.owns(j)) continue;
                const double sc = a.atol + fabs(y0d[blk][j]) * a.rtol;
                const double r = (static_cast<double>(k2[blk][j]) - static_cast<double>(k1[blk][j])) / sc;
                s2 += r * r;
            }
        const double d2 = sqrt(warp_sum(s2) / dim) / h0;
        const double h1 = (d1 <= 1e-15 && d2 <= 1e-15) ? fmax(1e-6, h0 * 1e-3) : pow(0.01 / fmax(d1, d2), 0.2);
        double dt_next = fmin(100.0 * h0, h1);
        double t = status == PB_TRAJ_OK ? a.t0 : a.t1;
        int64_t steps = 0;

        while (t < a.t1 && steps < a.max_steps) {
            ++steps;
            double dt = dt_next;
            if (t + dt > a.t1) dt = a.t1 - t;
            if (dt <= 0.0) break;
            if (t + dt == t) {
                status = PB_TRAJ_DT_UNDERFLOW;
                break;
            }
            const R h = static_cast<R>(dt);
#define PB_NET_STAGE(expr)                            \
    _Pragma("unroll") for (int blk = 0; blk < 3; ++blk) \
        _Pragma("unroll") for (int j = 0; j < NPL; ++j) ys[blk][j] = y[blk][j] + h * (expr);
            PB_NET_STAGE(R(dp::a21) * k1[blk][j]);
            W.rhs(ys, k2);
            PB_NET_STAGE(R(dp::a31) * k1[blk][j] + R(dp::a32) * k2[blk][j]);
            W.rhs(ys, k3);
            PB_NET_STAGE(R(dp::a41) * k1[blk][j] + R(dp::a42) * k2[blk][j] + R(dp::a43) * k3[blk][j]);
            W.rhs(ys, k4);
            PB_NET_STAGE(R(dp::a51) * k1[blk][j] + R(dp::a52) * k2[blk][j] + R(dp::a53) * k3[blk][j] +
                         R(dp::a54) * k4[blk][j]);
            W.rhs(ys, k5);
            PB_NET_STAGE(R(dp::a61) * k1[blk][j] + R(dp::a62) * k2[blk][j] + R(dp::a63) * k3[blk][j] +
                         R(dp::a64) * k4[blk][j] + R(dp::a65) * k5[blk][j]);
            W.rhs(ys, k6);
#undef PB_NET_STAGE
#pragma unroll
            for (int blk = 0; blk < 3; ++blk)
#pragma unroll
                for (int j = 0; j < NPL; ++j) {
                    d[blk][j] = h * (R(dp::b1) * k1[blk][j] + R(dp::b3) * k3[blk][j] + R(dp::b4) * k4[blk][j] +
                                     R(dp::b5) * k5[blk][j] + R(dp::b6) * k6[blk][j]);
                    yn[blk][j] = y[blk][j] + d[blk][j];
                }
            W.rhs(yn, k7);
            double e2 = 0.0;
#pragma unroll
            for (int blk = 0; blk < 3; ++blk)
#pragma unroll
                for (int j = 0; j < NPL; ++j) {
                    if (!W.owns(j)) continue;
                    const double e = static_cast<double>(
                        h * (R(dp::e1) * k1[blk][j] + R(dp::e3) * k3[blk][j] + R(dp::e4) * k4[blk][j] +
                             R(dp::e5) * k5[blk][j] + R(dp::e6) * k6[blk][j] + R(dp::e7) * k7[blk][j]));
                    const double sc = a.atol + a.rtol * fmax(fabs(static_cast<double>(y[blk][j])),
                                                             fabs(static_cast<double>(yn[blk][j])));
                    const double r = e / sc;
                    e2 += r * r;
                }
            const double err = sqrt(warp_sum(e2) / dim);
            if (!isfinite(err)) {
                status = PB_TRAJ_NONFINITE;
                break;
            }
            const bool accept = err <= 1.0;
            if (accept) {
                double m = 0.0;
#pragma unroll
                for (int blk = 0; blk < 3; ++blk)
#pragma unroll
                    for (int j = 0; j < NPL; ++j) {
                        if (mixed) {
                            const R corr = d[blk][j] - yc[blk][j];
                            const R nv = y[blk][j] + corr;
                            yc[blk][j] = (nv - y[blk][j]) - corr;
                            y[blk][j] = nv;
                        } else {
                            y[blk][j] = yn[blk][j];
                        }
                        k1[blk][j] = k7[blk][j];
                        if (W.owns(j)) m = fmax(m, fabs(static_cast<double>(y[blk][j])));
                    }
                t += dt;
                if (a.unbounded_thr > 0.0 && warp_max(m) >= a.unbounded_thr) {
                    status = PB_TRAJ_UNBOUNDED;
                    break;
                }
            }
            const double fac = (err == 0.0) ? dp::max_factor
                                            : fmin(dp::max_factor, fmax(accept ? 1.0 : dp::min_factor,
                                                                        dp::safety * pow(err, -0.2)));
            dt_next = dt * fac;
        }
        if (status == PB_TRAJ_OK && t < a.t1 && steps >= a.max_steps) status = PB_TRAJ_MAX_STEPS;

        // synchronisation features at the final state (+inf after an unbounded stop)
        double dev[3];
#pragma unroll
        for (int blk = 0; blk < 3; ++blk) {
            double mx = -CUDART_INF, mn = CUDART_INF;
#pragma unroll
            for (int j = 0; j < NPL; ++j)
                if (W.owns(j)) {
                    mx = fmax(mx, static_cast<double>(y[blk][j]));
                    mn = fmin(mn, static_cast<double>(y[blk][j]));
                }
            dev[blk] = (status == PB_TRAJ_UNBOUNDED) ? CUDART_INF : warp_max(mx) - warp_min(mn);
        }
        if (lane == 0) {
            for (int c = 0; c < a.n_features && a.features_out; ++c) {
                const int st = a.feat_state[c];
                double v = CUDART_NAN;
                if (a.feat_kind[c] == PB_FEAT_SYNC_DEV)
                    v = st == 3 ? fmax(dev[0], fmax(dev[1], dev[2])) : (st >= 0 && st < 3 ? dev[st] : CUDART_NAN);
                a.features_out[traj * a.n_features + c] = v;
            }
            if (a.status_out) a.status_out[traj] = status;
            if (a.steps_out) a.steps_out[traj] = steps;
        }
        if (a.y_final_out) {
#pragma unroll
            for (int blk = 0; blk < 3; ++blk)
#pragma unroll
                for (int j = 0; j < NPL; ++j) {
                    if (!W.owns(j)) continue;
                    const int64_t idx = traj * a.dim + blk * n_nodes + lane + 32 * j;
                    if (a.y_out_dtype == PB_DTYPE_F64)
                        static_cast<double*>(a.y_final_out)[idx] = static_cast<double>(y[blk][j]);
                    else
                        static_cast<float*>(a.y_final_out)[idx] = static_cast<float>(y[blk][j]);
                }
        }
        __syncwarp();
    }
}

}  // namespace pb
