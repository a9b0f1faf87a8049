// Surrogate MLP kernels: BF16 tensor-core GEMM with fused epilogues, GELU
// backward, softmax cross-entropy, bias gradient, AdamW, casts, and the
// confidence gate that routes uncertain ICs back to the integrator.
//
// The surrogate maps (initial condition, parameters) to attractor-class
// probabilities; it is trained on labels the integrator itself produced.  It
// has no counterpart in the reference.
//
// GEMM: C[m,n] = alpha * sum_k A(m,k) B(k,n) (+ bias[n]) with an optional GELU,
// A and B addressed through arbitrary element strides so the same kernel serves
// the forward (X W^T), the input gradient (dZ W) and the weight gradient
// (dZ^T X) without transposed copies.  64x64 block tile, k-tile 32, 4 warps of
// 32x32, mma.sync m16n8k16 BF16 x BF16 -> FP32.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <math_constants.h>
#include <stdint.h>

#include "pb_gelu.cuh"
#include "pybasin_b200.h"

namespace {

constexpr int BM = 64, BN = 64, BK = 32, PADK = 8;

__device__ __forceinline__ void mma_bf16_16816(float (&c)[4], const uint32_t (&a)[4], const uint32_t (&b)[2])
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
        "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

using pb::gelu;
using pb::gelu_grad;

template <int EPI>  // 0: none, 1: GELU
__global__ void __launch_bounds__(128) k_gemm_bf16(const __nv_bfloat16* __restrict__ A, int64_t sam, int64_t sak,
                                                   const __nv_bfloat16* __restrict__ B, int64_t sbk, int64_t sbn,
                                                   const float* __restrict__ bias, float alpha, int M, int N, int K,
                                                   float* __restrict__ Cf, __nv_bfloat16* __restrict__ Cb,
                                                   float* __restrict__ Zpre, int64_t ldc)
{
    __shared__ __align__(16) __nv_bfloat16 As[BM][BK + PADK];
    __shared__ __align__(16) __nv_bfloat16 Bs[BN][BK + PADK];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
    const int g = lane >> 2, tg = lane & 3;
    float acc[2][4][4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int r = 0; r < 4; ++r) acc[i][j][r] = 0.f;

    const __nv_bfloat16 zero = __float2bfloat16(0.f);
    for (int k0 = 0; k0 < K; k0 += BK) {
        // stage A (BM x BK) and B^T (BN x BK): 2048 elements each, 16 per thread
        for (int e = tid; e < BM * BK; e += 128) {
            const int r = e / BK, c = e % BK;
            const int gm = m0 + r, gk = k0 + c;
            As[r][c] = (gm < M && gk < K) ? A[gm * sam + gk * sak] : zero;
        }
        for (int e = tid; e < BN * BK; e += 128) {
            const int r = e / BK, c = e % BK;
            const int gn = n0 + r, gk = k0 + c;
            Bs[r][c] = (gn < N && gk < K) ? B[gk * sbk + gn * sbn] : zero;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < BK; kk += 16) {
            uint32_t af[2][4], bf[4][2];
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                const int r = wm + i * 16 + g;
                af[i][0] = *reinterpret_cast<const uint32_t*>(&As[r][kk + 2 * tg]);
                af[i][1] = *reinterpret_cast<const uint32_t*>(&As[r + 8][kk + 2 * tg]);
                af[i][2] = *reinterpret_cast<const uint32_t*>(&As[r][kk + 2 * tg + 8]);
                af[i][3] = *reinterpret_cast<const uint32_t*>(&As[r + 8][kk + 2 * tg + 8]);
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int n = wn + j * 8 + g;
                bf[j][0] = *reinterpret_cast<const uint32_t*>(&Bs[n][kk + 2 * tg]);
                bf[j][1] = *reinterpret_cast<const uint32_t*>(&Bs[n][kk + 2 * tg + 8]);
            }
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) mma_bf16_16816(acc[i][j], af[i], bf[j]);
        }
        __syncthreads();
    }
    // epilogue: alpha, bias, optional pre-activation copy, activation, store
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const int m = m0 + wm + i * 16 + g + (r >= 2 ? 8 : 0);
                const int n = n0 + wn + j * 8 + 2 * tg + (r & 1);
                if (m >= M || n >= N) continue;
                float v = alpha * acc[i][j][r];
                if (bias) v += bias[n];
                if (Zpre) Zpre[m * ldc + n] = v;
                if (EPI == 1) v = gelu(v);
                if (Cf) Cf[m * ldc + n] = v;
                if (Cb) Cb[m * ldc + n] = __float2bfloat16(v);
            }
}

// dZ = dY * gelu'(Z), written as BF16 (and optionally FP32)
__global__ void k_gelu_backward(const float* __restrict__ dy, const float* __restrict__ z, int64_t n,
                                __nv_bfloat16* __restrict__ dzb, float* __restrict__ dzf)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float v = dy[i] * gelu_grad(z[i]);
        if (dzb) dzb[i] = __float2bfloat16(v);
        if (dzf) dzf[i] = v;
    }
}

// softmax cross-entropy over rows of logits (M x C): loss_sum += -log p[y],
// dlogits = (p - onehot) * scale (BF16 + FP32 copies, either may be NULL)
__global__ void k_softmax_xent(const float* __restrict__ logits, const int32_t* __restrict__ y, int M, int C,
                               float scale, __nv_bfloat16* __restrict__ dzb, float* __restrict__ dzf,
                               float* __restrict__ loss_sum, int32_t* __restrict__ correct)
{
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= M) return;
    const float* l = logits + (int64_t)m * C;
    float mx = -CUDART_INF_F;
    int arg = 0;
    for (int c = 0; c < C; ++c)
        if (l[c] > mx) {
            mx = l[c];
            arg = c;
        }
    float s = 0.f;
    for (int c = 0; c < C; ++c) s += __expf(l[c] - mx);
    const int yc = y ? y[m] : -1;
    for (int c = 0; c < C; ++c) {
        const float p = __expf(l[c] - mx) / s;
        const float g = (p - (c == yc ? 1.f : 0.f)) * scale;
        if (dzb) dzb[(int64_t)m * C + c] = __float2bfloat16(g);
        if (dzf) dzf[(int64_t)m * C + c] = g;
    }
    if (yc >= 0 && yc < C) {
        if (loss_sum) atomicAdd(loss_sum, -(l[yc] - mx - __logf(s)));
        if (correct && arg == yc) atomicAdd(correct, 1);
    }
}

// db[n] = alpha * sum_m dZ[m, n]
__global__ void k_bias_grad(const float* __restrict__ dz, int M, int N, float alpha, float* __restrict__ db)
{
    const int n = blockIdx.x;
    float s = 0.f;
    for (int m = threadIdx.x; m < M; m += blockDim.x) s += dz[(int64_t)m * N + n];
    __shared__ float red[256];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) db[n] = alpha * red[0];
}

// AdamW on FP32 master weights, refreshing the BF16 copy
__global__ void k_adamw(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m1,
                        float* __restrict__ m2, __nv_bfloat16* __restrict__ wb, int64_t n, float lr, float b1, float b2,
                        float eps, float wd, float bc1, float bc2)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float a = b1 * m1[i] + (1.f - b1) * gi;
        const float b = b2 * m2[i] + (1.f - b2) * gi * gi;
        m1[i] = a;
        m2[i] = b;
        float wi = w[i] * (1.f - lr * wd);
        wi -= lr * (a / bc1) / (sqrtf(b / bc2) + eps);
        w[i] = wi;
        if (wb) wb[i] = __float2bfloat16(wi);
    }
}

__global__ void k_cast_bf16(const float* __restrict__ x, __nv_bfloat16* __restrict__ y, int64_t n)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        y[i] = __float2bfloat16(x[i]);
}

// Inputs of the surrogate: z = (x - shift) * scale per column of x = (IC, FP64
// parameter row), then for each of the n_freq rows f of `freq` (cycles per unit
// of z) the pair sin(2 pi f.z), cos(2 pi f.z) (random Fourier features, which let
// a small MLP resolve finely interleaved basins); written as BF16 rows
// [z, sin, cos] (n x d_pad, zero padded).
constexpr int kMaxRawInputs = 16;

// A block takes R = 256 / U rows at a time (U = max(n_freq, 1) threads per row):
// the frequencies and the rows' z-scored columns are staged in shared memory, then
// thread (r, j) writes frequency j's sine-cosine pair of row r and every U-th z or
// padding column from j on, so neighbouring threads write neighbouring columns.
// Dynamic shared memory: (n_freq + R) * d floats.
__global__ void __launch_bounds__(256) k_features_in(const float* __restrict__ ic, int S,
                                                     const double* __restrict__ prm, int np,
                                                     const int32_t* __restrict__ prow, int64_t n_rows,
                                                     const float* __restrict__ shift,
                                                     const float* __restrict__ scale,
                                                     const float* __restrict__ freq, int n_freq, int64_t n,
                                                     int d_pad, __nv_bfloat16* __restrict__ out)
{
    extern __shared__ float fsm[];
    const int d = S + np;
    const int U = n_freq > 0 ? n_freq : 1;
    const int R = 256 / U;
    float* f_s = fsm;               // n_freq x d
    float* z_s = fsm + n_freq * d;  // R x d
    for (int i = threadIdx.x; i < n_freq * d; i += blockDim.x) f_s[i] = freq[i];
    const int n_zero = d_pad - d - 2 * n_freq;
    const int r_loc = threadIdx.x / U, j = threadIdx.x - r_loc * U;
    for (int64_t r0 = static_cast<int64_t>(blockIdx.x) * R; r0 < n; r0 += static_cast<int64_t>(gridDim.x) * R) {
        __syncthreads();  // the previous rows' z are consumed
        for (int i = threadIdx.x; i < R * d; i += blockDim.x) {
            const int rr = i / d, c = i - rr * d;
            const int64_t r = r0 + rr;
            float v = 0.f;
            if (r < n) {
                if (c < S) {
                    v = ic[r * S + c];
                } else {
                    // the IC's own parameter row (prow), else row 0; a row index out of
                    // range gives NaN inputs, whose logits the gate routes to the integrator
                    const int64_t q = prow ? static_cast<int64_t>(prow[r]) : 0;
                    v = (q >= 0 && q < n_rows) ? static_cast<float>(prm[q * np + (c - S)]) : CUDART_NAN_F;
                }
            }
            z_s[i] = (v - shift[c]) * scale[c];
        }
        __syncthreads();
        const int64_t r = r0 + r_loc;
        if (r_loc >= R || r >= n) continue;
        const float* z = z_s + r_loc * d;
        __nv_bfloat16* o = out + r * d_pad;
        if (n_freq > 0) {
            float turns = 0.f;
            for (int c = 0; c < d; ++c) turns = fmaf(f_s[j * d + c], z[c], turns);
            // sin and cos of 2 pi turns: the whole turns taken off exactly (|turns| <
            // 2^22), the rest, in [-pi, pi], to the hardware sine and cosine (absolute
            // error about 2^-21, far below the BF16 step of the result)
            float sn, cs;
            __sincosf(6.28318530717958648f * (turns - rintf(turns)), &sn, &cs);
            o[d + j] = __float2bfloat16(sn);
            o[d + n_freq + j] = __float2bfloat16(cs);
        }
        for (int c = j; c < d; c += U) o[c] = __float2bfloat16(z[c]);
        for (int c = j; c < n_zero; c += U) o[d + 2 * n_freq + c] = __float2bfloat16(0.f);
    }
}

// Confidence gate: softmax over C logits per row; rows with max probability
// >= threshold keep the surrogate's class, the others (and every audited row)
// are appended to `route` for integration.  label = argmax, conf = max prob.
__global__ void k_gate(const float* __restrict__ logits, int64_t n, int C, float threshold,
                       const uint8_t* __restrict__ audit, int32_t* __restrict__ label, float* __restrict__ conf,
                       int32_t* __restrict__ route, int32_t* __restrict__ n_route)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* l = logits + i * C;
    float mx = -CUDART_INF_F;
    int arg = 0;
    for (int c = 0; c < C; ++c)
        if (l[c] > mx) {
            mx = l[c];
            arg = c;
        }
    float s = 0.f;
    for (int c = 0; c < C; ++c) s += __expf(l[c] - mx);
    const float p = 1.f / s;
    label[i] = arg;
    if (conf) conf[i] = p;
    const bool aud = audit && audit[i];
    if (!(p >= threshold) || aud) {  // a non-finite confidence is routed too
        const int pos = atomicAdd(n_route, 1);
        route[pos] = static_cast<int32_t>(i);
    }
}

// y[k] = x[idx[k]] for rows of width w (gather of routed ICs)
__global__ void k_gather_rows(const float* __restrict__ x, int w, const int32_t* __restrict__ idx,
                              const int32_t* __restrict__ n_idx, int64_t max_rows, float* __restrict__ y)
{
    const int64_t n = min(static_cast<int64_t>(*n_idx), max_rows);
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n * w;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = e / w;
        const int c = static_cast<int>(e - k * w);
        y[e] = x[(int64_t)idx[k] * w + c];
    }
}

// merge: out[idx[k]] = integrated[k] for routed rows, counts per class
__global__ void k_merge_labels(const int32_t* __restrict__ integ, const int32_t* __restrict__ idx,
                               const int32_t* __restrict__ n_idx, int64_t max_rows, int32_t* __restrict__ label,
                               int32_t* __restrict__ surrogate_label_of_routed)
{
    const int64_t n = min(static_cast<int64_t>(*n_idx), max_rows);
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        const int i = idx[k];
        if (surrogate_label_of_routed) surrogate_label_of_routed[k] = label[i];
        label[i] = integ[k];
    }
}

// Per-class counts of the final labels, and the audit tally over the routed rows:
// stats[0] audited rows, stats[1] of those the ones the surrogate was confident
// about (conf >= threshold), stats[2] of those the ones the integrator labelled
// differently.  counts and stats start at zero (cleared by the entry point).
constexpr int kMaxSummaryClasses = 64;
__global__ void k_gate_summary(const int32_t* __restrict__ label, int64_t n, int C, const int32_t* __restrict__ route,
                               const int32_t* __restrict__ n_route, int64_t max_rows, const uint8_t* __restrict__ audit,
                               const float* __restrict__ conf, float threshold, const int32_t* __restrict__ sur,
                               const int32_t* __restrict__ integ, unsigned long long* __restrict__ counts,
                               int32_t* __restrict__ stats)
{
    __shared__ unsigned int hist[kMaxSummaryClasses];
    __shared__ int tally[3];
    for (int c = threadIdx.x; c < C; c += blockDim.x) hist[c] = 0u;
    if (threadIdx.x < 3) tally[threadIdx.x] = 0;
    __syncthreads();
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += stride) {
        const int c = label[i];
        if (c >= 0 && c < C) atomicAdd(&hist[c], 1u);
    }
    const int64_t k = route ? min(static_cast<int64_t>(*n_route), max_rows) : 0;
    int na = 0, nc = 0, nd = 0;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < k; q += stride) {
        const int i = route[q];
        if (audit && audit[i]) {
            ++na;
            if (conf[i] >= threshold) {
                ++nc;
                nd += sur[q] != integ[q] ? 1 : 0;
            }
        }
    }
    if (na) atomicAdd(&tally[0], na);
    if (nc) atomicAdd(&tally[1], nc);
    if (nd) atomicAdd(&tally[2], nd);
    __syncthreads();
    for (int c = threadIdx.x; c < C; c += blockDim.x)
        if (hist[c]) atomicAdd(&counts[c], static_cast<unsigned long long>(hist[c]));
    if (threadIdx.x < 3 && tally[threadIdx.x]) atomicAdd(&stats[threadIdx.x], tally[threadIdx.x]);
}

int grid_for(int64_t n, int block)
{
    int64_t g = (n + block - 1) / block;
    if (g > 65535LL * 16) g = 65535LL * 16;
    return static_cast<int>(g < 1 ? 1 : g);
}

int map_err(cudaError_t e) { return e == cudaSuccess ? PB_SUCCESS : PB_ECUDA; }

}  // namespace

extern "C" {

int pb_mlp_gemm(const void* A, int64_t sam, int64_t sak, const void* B, int64_t sbk, int64_t sbn, const float* bias,
                float alpha, int32_t M, int32_t N, int32_t K, int32_t gelu, float* c_f32, void* c_bf16,
                float* z_pre, int64_t ldc, void* stream)
{
    if (!A || !B || M < 0 || N < 0 || K < 0 || (!c_f32 && !c_bf16 && !z_pre)) return PB_EINVAL;
    if (M == 0 || N == 0) return PB_SUCCESS;
    dim3 grid((N + BN - 1) / BN, (M + BM - 1) / BM);
    if (grid.y > 65535) return PB_EINVAL;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    auto a = static_cast<const __nv_bfloat16*>(A);
    auto b = static_cast<const __nv_bfloat16*>(B);
    auto cb = static_cast<__nv_bfloat16*>(c_bf16);
    if (gelu)
        k_gemm_bf16<1><<<grid, 128, 0, st>>>(a, sam, sak, b, sbk, sbn, bias, alpha, M, N, K, c_f32, cb, z_pre, ldc);
    else
        k_gemm_bf16<0><<<grid, 128, 0, st>>>(a, sam, sak, b, sbk, sbn, bias, alpha, M, N, K, c_f32, cb, z_pre, ldc);
    return map_err(cudaGetLastError());
}

int pb_mlp_gelu_backward(const float* dy, const float* z, int64_t n, void* dz_bf16, float* dz_f32, void* stream)
{
    if (!dy || !z || n < 0) return PB_EINVAL;
    if (n == 0) return PB_SUCCESS;
    k_gelu_backward<<<grid_for(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        dy, z, n, static_cast<__nv_bfloat16*>(dz_bf16), dz_f32);
    return map_err(cudaGetLastError());
}

int pb_mlp_softmax_xent(const float* logits, const int32_t* labels, int32_t M, int32_t C, float scale, void* dz_bf16,
                        float* dz_f32, float* loss_sum, int32_t* correct, void* stream)
{
    if (!logits || M < 0 || C <= 0) return PB_EINVAL;
    if (M == 0) return PB_SUCCESS;
    k_softmax_xent<<<(M + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        logits, labels, M, C, scale, static_cast<__nv_bfloat16*>(dz_bf16), dz_f32, loss_sum, correct);
    return map_err(cudaGetLastError());
}

int pb_mlp_bias_grad(const float* dz, int32_t M, int32_t N, float alpha, float* db, void* stream)
{
    if (!dz || !db || M < 0 || N <= 0) return PB_EINVAL;
    k_bias_grad<<<N, 256, 0, static_cast<cudaStream_t>(stream)>>>(dz, M, N, alpha, db);
    return map_err(cudaGetLastError());
}

int pb_mlp_adamw(float* w, const float* g, float* m1, float* m2, void* w_bf16, int64_t n, float lr, float beta1,
                 float beta2, float eps, float weight_decay, int32_t step, void* stream)
{
    if (!w || !g || !m1 || !m2 || n < 0 || step < 1) return PB_EINVAL;
    if (n == 0) return PB_SUCCESS;
    const float bc1 = 1.f - powf(beta1, static_cast<float>(step));
    const float bc2 = 1.f - powf(beta2, static_cast<float>(step));
    k_adamw<<<grid_for(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        w, g, m1, m2, static_cast<__nv_bfloat16*>(w_bf16), n, lr, beta1, beta2, eps, weight_decay, bc1, bc2);
    return map_err(cudaGetLastError());
}

int pb_mlp_cast_bf16(const float* x, void* y, int64_t n, void* stream)
{
    if (!x || !y || n < 0) return PB_EINVAL;
    if (n == 0) return PB_SUCCESS;
    k_cast_bf16<<<grid_for(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(x, static_cast<__nv_bfloat16*>(y),
                                                                                  n);
    return map_err(cudaGetLastError());
}

int pb_surrogate_inputs_rows(const float* ic, int32_t S, const double* params, int64_t n_param_rows,
                             int32_t n_params, const int32_t* param_index, const float* shift, const float* scale,
                             const float* freq, int32_t n_freq, int64_t n, int32_t d_pad, void* out_bf16,
                             void* stream)
{
    if (!ic || !shift || !scale || !out_bf16 || S <= 0 || n_params < 0 || n_freq < 0 ||
        S + n_params > kMaxRawInputs || S + n_params + 2 * n_freq > d_pad || n < 0 || n_param_rows < 0)
        return PB_EINVAL;
    if ((n_params > 0 && (!params || n_param_rows < 1)) || (n_freq > 0 && !freq)) return PB_EINVAL;
    if (n == 0) return PB_SUCCESS;
    if (n_freq > 128) return PB_EINVAL;  // at least two rows per 256-thread block
    const int U = n_freq > 0 ? n_freq : 1, R = 256 / U;
    const size_t fsmem = static_cast<size_t>(n_freq + R) * (S + n_params) * sizeof(float);
    // a grid of 16 blocks per SM strides over the rows (each block stages the
    // frequencies once)
    const int64_t blocks = (n + R - 1) / R;
    k_features_in<<<static_cast<unsigned>(blocks < 148 * 16 ? blocks : 148 * 16), 256, fsmem,
                    static_cast<cudaStream_t>(stream)>>>(
        ic, S, params, n_params, param_index, n_param_rows, shift, scale, freq, n_freq, n, d_pad,
        static_cast<__nv_bfloat16*>(out_bf16));
    return map_err(cudaGetLastError());
}

int pb_surrogate_inputs(const float* ic, int32_t S, const double* params, int32_t n_params, const float* shift,
                        const float* scale, const float* freq, int32_t n_freq, int64_t n, int32_t d_pad,
                        void* out_bf16, void* stream)
{
    return pb_surrogate_inputs_rows(ic, S, params, 1, n_params, nullptr, shift, scale, freq, n_freq, n, d_pad,
                                    out_bf16, stream);
}

int pb_surrogate_gate(const float* logits, int64_t n, int32_t C, float threshold, const uint8_t* audit,
                      int32_t* label, float* conf, int32_t* route, int32_t* n_route, void* stream)
{
    if (!logits || !label || !route || !n_route || C <= 0 || n < 0) return PB_EINVAL;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemsetAsync(n_route, 0, sizeof(int32_t), st);
    if (e != cudaSuccess) return PB_ECUDA;
    if (n == 0) return PB_SUCCESS;
    k_gate<<<static_cast<unsigned>((n + 255) / 256), 256, 0, st>>>(logits, n, C, threshold, audit, label, conf, route,
                                                                     n_route);
    return map_err(cudaGetLastError());
}

int pb_gather_rows(const float* x, int32_t width, const int32_t* idx, const int32_t* n_idx, int64_t max_rows, float* y,
                   void* stream)
{
    if (!x || !idx || !n_idx || !y || width <= 0 || max_rows < 0) return PB_EINVAL;
    if (max_rows == 0) return PB_SUCCESS;
    k_gather_rows<<<grid_for(max_rows * width, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        x, width, idx, n_idx, max_rows, y);
    return map_err(cudaGetLastError());
}

int pb_gate_summary(const int32_t* label, int64_t n, int32_t C, const int32_t* route, const int32_t* n_route,
                    int64_t max_rows, const uint8_t* audit, const float* conf, float threshold,
                    const int32_t* surrogate_label_of_routed, const int32_t* integrated, int64_t* counts,
                    int32_t* stats, void* stream)
{
    if (!label || n < 0 || C <= 0 || C > kMaxSummaryClasses || !counts || !stats || max_rows < 0) return PB_EINVAL;
    if (route && (!n_route || !conf || !surrogate_label_of_routed || !integrated)) return PB_EINVAL;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (cudaMemsetAsync(counts, 0, sizeof(int64_t) * C, st) != cudaSuccess ||
        cudaMemsetAsync(stats, 0, sizeof(int32_t) * 3, st) != cudaSuccess)
        return PB_ECUDA;
    const int64_t work = n > max_rows ? n : max_rows;
    if (work == 0) return PB_SUCCESS;
    int blocks = grid_for(work, 256);
    if (blocks > 1184) blocks = 1184;  // 8 blocks per SM of a 148-SM part: one atomic flush each
    k_gate_summary<<<blocks, 256, 0, st>>>(label, n, C, route, n_route, max_rows, audit, conf, threshold,
                                           surrogate_label_of_routed, integrated,
                                           reinterpret_cast<unsigned long long*>(counts), stats);
    return map_err(cudaGetLastError());
}

int pb_merge_labels(const int32_t* integrated, const int32_t* idx, const int32_t* n_idx, int64_t max_rows,
                    int32_t* label, int32_t* surrogate_label_of_routed, void* stream)
{
    if (!integrated || !idx || !n_idx || !label || max_rows < 0) return PB_EINVAL;
    if (max_rows == 0) return PB_SUCCESS;
    k_merge_labels<<<grid_for(max_rows, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        integrated, idx, n_idx, max_rows, label, surrogate_label_of_routed);
    return map_err(cudaGetLastError());
}

}  // extern "C"
