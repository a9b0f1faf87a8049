// Surrogate training on the 5th-generation tensor cores.
//
// One training step of the surrogate MLP (minibatch of B rows, layers of
// K_l -> N_l units) is three kinds of GEMM, all served by k_gemm_tc:
//
//   forward       Z_l  = X_l W_l^T + b_l        (M = B,   N = N_l, K = K_l)
//                 X_l+1 = GELU(Z_l) in BF16, Z_l kept in FP32 for the backward pass
//   input grad    dZ_l-1 = (dZ_l W_l) * GELU'(Z_l-1) in BF16, with the column sums
//                 of dZ_l-1 (the bias gradient) as per-warp partials
//                                              (M = B,   N = K_l, K = N_l)
//   weight grad   dW_l = dZ_l^T X_l, split over the batch into partials
//                                              (M = N_l, N = K_l, K = B)
//
// Every operand is read from global memory through element strides and staged
// into shared memory in the K-major core-matrix layout of tcgen05.mma (8 rows x
// 16 bytes per core matrix, core (row/8, k/8) at ((row/8) * (KC/8) + k/8) * 128
// bytes).  An operand contiguous along K, with rows and K multiples of 8 and
// 16-byte aligned rows, is brought in by one TMA copy: a 4-D tensor map over
// (k mod 8, row mod 8, k / 8, row / 8) with strides (2 B, row pitch, 16 B, 8 row
// pitches), whose box lands in shared memory in exactly the core-matrix order.
// Other K-contiguous operands are copied with cp.async, 16 bytes (8 k) at a time;
// one contiguous along its rows is read 16 bytes (8 rows) at a time and
// scattered to the 8 core rows.  The
// training step keeps every operand K-contiguous: the producers of the
// activations and of dZ also write transposed copies (one row of the copy per
// column, consecutive threads writing consecutive elements), the optimiser
// writes W^T next to W, and the epoch's shuffle writes the inputs transposed.
// A CTA owns a 128-row tile of C and `bn` of its columns (one tcgen05.mma per 16
// of K, M = 128, N = bn, BF16 x BF16 -> FP32 in tensor memory), and a K chunk of
// at most 256 (the weight gradient splits the batch into chunks; its partials
// are summed by the optimiser in a fixed order, so a step is deterministic).
// The epilogue reads the accumulator with tcgen05.ld, one TMEM lane (one row
// of C) per thread.
//
// The softmax cross-entropy writes dZ of the last layer and its bias partials;
// k_adamw_multi updates every parameter tensor of the network in one launch,
// summing each gradient's partials first and refreshing the BF16 copies.  The
// whole step allocates nothing, so a training run can be captured as one CUDA
// graph and replayed.
//
// Every mbarrier wait is bounded: on a timeout the CTA sets the error flag,
// frees its tensor memory and returns.  There is no counterpart in the
// reference (its surrogate-free pipeline has no learned part).
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <math_constants.h>
#include <stdint.h>

#include <atomic>
#include <cstdlib>
#include <mutex>

#include "pb_gelu.cuh"
#include "pybasin_b200.h"

namespace {

constexpr int kRows = 128;             // MMA M = rows of a CTA tile = TMEM lanes
constexpr int kThreads = 256;          // 8 warps: TMEM lane quarter w % 4, column chunks from 32 (w / 4)
constexpr int kMaxKc = 256;            // K of one CTA (split-K chunk)
constexpr int kMaxBn = 256;            // N of one CTA
constexpr long long kWaitPolls = 1ll << 22;
constexpr int kMaxSeg = 16;            // parameter tensors of one AdamW launch
constexpr int kMaxSmem = 227 * 1024;   // dynamic shared memory of one CTA

struct GemmTcArgs {
    const __nv_bfloat16* A;  // A(m, k) = A[m * sam + k * sak]
    const __nv_bfloat16* B;  // B(n, k) = B[n * sbn + k * sbk]   (C = A B^T)
    int64_t sam, sak, sbn, sbk;
    int M, N, K;
    int kc;    // K per CTA: multiple of 16, <= 256; blockIdx.z takes K range [z kc, (z+1) kc)
    int bn;    // N per CTA: multiple of 16, <= 256
    int mode;  // PB_TRAIN_*
    const float* bias;       // forward: (N)
    const float* z_in;       // input gradient: pre-activations of the layer below, (M, ldz)
    int64_t ldz;
    float* out_f32;          // forward linear: (M, ldc); weight grad: partial z at z * M * ldc
    __nv_bfloat16* out_bf16; // forward GELU, input grad: (M, ldc)
    __nv_bfloat16* out_t;    // forward GELU, input grad: the same transposed, out_t[n * ldt + m], optional
    float* z_pre;            // forward GELU: (M, ldc), optional
    float* col_part;         // input grad: (gridDim.x * 4, ldp) column partial sums, optional
    int64_t ldc, ldt, ldp;
    int* error;
    int zin_off;  // input gradient: the z_in tile, loaded while the MMAs run
    int bar_off;  // the mbarriers and the tensor-memory slot
    int tma_a, tma_b;  // operand brought in by its tensor map (else cp.async / scatter)
};

// Shared memory of one CTA: the operand tiles (A 128 x kc, B bn x kc), then for
// the input gradient the z_in tile (FP32, pitch bn + 4: rows shifted by 16 bytes,
// so a thread per row reads conflict-free), then the barrier.
__host__ __device__ inline int tile_f32_bytes(int bn) { return kRows * (bn + 4) * 4; }
__host__ __device__ inline int align16i(int v) { return (v + 15) & ~15; }
inline void smem_plan(int mode, int kc, int bn, int* zin_off, int* bar_off, int* total)
{
    int off = align16i(kRows * kc * 2 + bn * kc * 2);
    *zin_off = off;
    if (mode == PB_TRAIN_DX) off += tile_f32_bytes(bn);
    *bar_off = off;
    *total = off + 64;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint32_t core_offset(int row, int k, int K)
{
    return ((static_cast<uint32_t>(row >> 3) * static_cast<uint32_t>(K >> 3) + static_cast<uint32_t>(k >> 3)) << 7) +
           (static_cast<uint32_t>(row & 7) << 4) + (static_cast<uint32_t>(k & 7) << 1);
}

// shared-memory matrix descriptor: start, leading (K-direction core stride) and
// stride (8-row-group stride) byte offsets in 16-byte units, version 1, no swizzle
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    return static_cast<uint64_t>((addr >> 4) & 0x3FFFu) | (static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16) |
           (static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// kind::f16 instruction descriptor: FP32 accumulator, BF16 A and B, both K-major
__device__ __forceinline__ uint32_t instr_desc(int M, int N)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(N >> 3) << 17) |
           (static_cast<uint32_t>(M >> 4) << 24);
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity)
{
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    return done != 0;
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity)
{
    for (long long i = 0; i < kWaitPolls; ++i)
        if (mbar_try(bar, parity)) return true;
    return false;
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

// One tile of an operand by its 4-D tensor map: coordinates (k mod 8 = 0, row mod 8
// = 0, k0 / 8, row0 / 8); completes on the mbarrier with the box's byte count.
__device__ __forceinline__ void tma_load_tile(uint32_t dst, const CUtensorMap* map, int k0, int row0, uint32_t bar)
{
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
        "[%6];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(0), "r"(0), "r"(k0 >> 3), "r"(row0 >> 3), "r"(bar)
        : "memory");
}

// The virtual row of ones (the bias column) of a TMA-staged B tile: the copy left
// it zero (it lies past the tensor map's rows), so it is written after the copy.
__device__ __forceinline__ void ones_row(uint8_t* s, int r, int KC, int k0, int kend)
{
    const __nv_bfloat16 zero = __float2bfloat16(0.f), one = __float2bfloat16(1.f);
    for (int kg = threadIdx.x; kg < (KC >> 3); kg += kThreads) {
        __align__(16) __nv_bfloat16 h[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) h[j] = k0 + kg * 8 + j < kend ? one : zero;
        *reinterpret_cast<uint4*>(s + core_offset(r, kg * 8, KC)) = *reinterpret_cast<const uint4*>(h);
    }
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc)
{
    const uint32_t mask0 = 0, mask1 = 0, mask2 = 0, mask3 = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(mask0), "r"(mask1), "r"(mask2), "r"(mask3));
}

__device__ __forceinline__ void mma_commit(uint32_t bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
          "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
          "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}

__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// The ragged cases of stage_row16 (a row past nrows, the ones row, a partial or
// unaligned group of 8 k): element by element, out of line (rare).
__device__ __noinline__ void stage_row16_slow(uint8_t* dst, const __nv_bfloat16* __restrict__ X, int64_t sr, int gr,
                                              int nrows, int gk, int kend, int ones_row)
{
    const __nv_bfloat16 zero = __float2bfloat16(0.f), one = __float2bfloat16(1.f);
    __align__(16) __nv_bfloat16 h[8];
    if (gr < nrows) {
        const __nv_bfloat16* src = X + static_cast<int64_t>(gr) * sr + gk;
        for (int j = 0; j < 8; ++j) h[j] = gk + j < kend ? src[j] : zero;
    } else {
        for (int j = 0; j < 8; ++j) h[j] = (gr == ones_row && gk + j < kend) ? one : zero;
    }
    *reinterpret_cast<uint4*>(dst) = *reinterpret_cast<const uint4*>(h);
}

// One 16-byte core row of a K-contiguous operand: row gr, k from gk (8 values),
// zero beyond nrows / kend, ones on ones_row; a cp.async when the group is whole.
__device__ __forceinline__ void stage_row16(uint8_t* dst, const __nv_bfloat16* __restrict__ X, int64_t sr, int gr,
                                            int nrows, int gk, int kend, int ones_row)
{
    const __nv_bfloat16* src = X + static_cast<int64_t>(gr) * sr + gk;
    if (gr < nrows && gk + 8 <= kend && aligned16(src))
        cp_async16(smem_u32(dst), src);
    else
        stage_row16_slow(dst, X, sr, gr, nrows, gk, kend, ones_row);
}

// Stage rows [row0, row0 + R) x k [k0, k0 + KC) of X(r, k) = X[r * sr + k * sk]
// (rows < nrows, k < kend valid, the rest zero) into the core-matrix layout at s.
// Row `ones_row` (>= nrows; -1 for none) reads 1 for every valid k: the column of
// ones whose product with the other operand is its column sums.  Copies from a
// K-contiguous operand are cp.async (completed by the caller's
// cp_async_wait_all); a row-contiguous operand is read eight 16-byte loads at a
// time (in flight together) and scattered.
__device__ __forceinline__ void stage_kcontig(uint8_t* s, const __nv_bfloat16* __restrict__ X, int64_t sr, int row0,
                                              int R, int nrows, int k0, int KC, int kend, int ones_row)
{
    // item i: row (i / 8 / groups) * 8 + i % 8, k group (i / 8) % groups.  Eight
    // consecutive threads fill one core matrix (128 contiguous bytes of shared
    // memory: no bank conflicts); a warp reads 64 contiguous bytes of 8 rows.
    const int groups = KC >> 3;
    for (int idx = threadIdx.x; idx < R * groups; idx += kThreads) {
        const int q = idx >> 3, rb = q / groups, kg = q - rb * groups;
        const int r = rb * 8 + (idx & 7);
        stage_row16(s + core_offset(r, kg * 8, KC), X, sr, row0 + r, nrows, k0 + kg * 8, kend, ones_row);
    }
}

__device__ __noinline__ void stage_rowcontig(uint8_t* s, const __nv_bfloat16* __restrict__ X, int64_t sr, int64_t sk,
                                             int row0, int R, int nrows, int k0, int KC, int kend, int ones_row)
{
    const __nv_bfloat16 zero = __float2bfloat16(0.f), one = __float2bfloat16(1.f);
    // contiguous along the rows (sr == 1): 8 rows of one k per 16-byte read, scattered
    // to the 8 core rows; consecutive threads take consecutive k
    const int total = (R >> 3) * KC;
    constexpr int kBatch = 8;
    for (int base = threadIdx.x; base < total; base += kThreads * kBatch) {
        uint4 v[kBatch];
#pragma unroll
        for (int u = 0; u < kBatch; ++u) {
            const int idx = base + u * kThreads;
            v[u] = make_uint4(0u, 0u, 0u, 0u);
            if (idx >= total) continue;
            const int rg = idx / KC, k = idx - rg * KC;
            const int gr = row0 + rg * 8, gk = k0 + k;
            if (gk >= kend) continue;
            const __nv_bfloat16* src = X + gr * sr + static_cast<int64_t>(gk) * sk;
            if (sr == 1 && gr + 8 <= nrows && aligned16(src)) {
                v[u] = *reinterpret_cast<const uint4*>(src);
            } else {
                __align__(16) __nv_bfloat16 h[8];
#pragma unroll
                for (int j = 0; j < 8; ++j)
                    h[j] = gr + j < nrows ? X[(gr + j) * sr + static_cast<int64_t>(gk) * sk]
                                          : (gr + j == ones_row ? one : zero);
                v[u] = *reinterpret_cast<const uint4*>(h);
            }
        }
#pragma unroll
        for (int u = 0; u < kBatch; ++u) {
            const int idx = base + u * kThreads;
            if (idx >= total) continue;
            const int rg = idx / KC, k = idx - rg * KC;
            const __nv_bfloat16* h = reinterpret_cast<const __nv_bfloat16*>(&v[u]);
#pragma unroll
            for (int j = 0; j < 8; ++j) *reinterpret_cast<__nv_bfloat16*>(s + core_offset(rg * 8 + j, k, KC)) = h[j];
        }
    }
}

using pb::gelu;
using pb::gelu_grad;

// Column sums of v[0..31] over the 32 lanes of the warp: afterwards lane j holds
// the sum of column j (a transposing butterfly: 31 shuffles for 32 columns).
__device__ __forceinline__ float warp_column_sums(float (&v)[32], int lane)
{
#pragma unroll
    for (int w = 16; w >= 1; w >>= 1) {
        const bool upper = (lane & w) != 0;
#pragma unroll
        for (int j = 0; j < w; ++j) {
            // keep columns of my half (lower half j, upper half j + w), send the others
            const float send = upper ? v[j] : v[j + w];
            const float keep = upper ? v[j + w] : v[j];
            v[j] = keep + __shfl_xor_sync(0xffffffffu, send, w);
        }
    }
    return v[0];
}

// MODE: the epilogue (PB_TRAIN_*); AK / BK: A / B contiguous along K (else along its rows)
// MODE: the epilogue (PB_TRAIN_*); AK / BK: A / B contiguous along K (else along its rows)
// Copy the [rows x cols] tile at t (pitch tp bytes, e-byte elements) to global
// dst (row stride ld elements): 16-byte pieces, consecutive threads along a row
// (coalesced), element by element where a piece is partial or unaligned.
template <int E>
__device__ __forceinline__ void tile_out(const uint8_t* t, int tp, uint8_t* dst, int64_t ld, int rows, int cols, int bn)
{
    const int per_row = bn * E / 16;
    for (int idx = threadIdx.x; idx < kRows * per_row; idx += kThreads) {
        const int r = idx / per_row, c = (idx - r * per_row) * (16 / E);
        if (r >= rows || c >= cols) continue;
        uint8_t* g = dst + (static_cast<int64_t>(r) * ld + c) * E;
        const uint8_t* sp = t + r * tp + c * E;
        if (c + 16 / E <= cols && aligned16(g)) {
            *reinterpret_cast<uint4*>(g) = *reinterpret_cast<const uint4*>(sp);
        } else {
            for (int j = 0; j < 16 / E && c + j < cols; ++j)
                for (int b = 0; b < E; ++b) g[j * E + b] = sp[j * E + b];
        }
    }
}

// MODE: the epilogue (PB_TRAIN_*); AK / BK: A / B contiguous along K (else along its rows)
template <int MODE, bool AK, bool BK>
__global__ void __launch_bounds__(kThreads, 1) k_gemm_tc(const GemmTcArgs p, const __grid_constant__ CUtensorMap map_a,
                                                          const __grid_constant__ CUtensorMap map_b)
{
    extern __shared__ __align__(1024) uint8_t smem[];
    const int KC = p.kc, BN = p.bn;
    uint8_t* As = smem;
    uint8_t* Bs = smem + kRows * KC * 2;
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + p.bar_off);  // [0] MMAs done, [1] TMA copies done
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bar + 2);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * kRows, n0 = blockIdx.y * BN, k0 = blockIdx.z * KC;
    const int kend = min(p.K, k0 + KC);
    const int rows = min(kRows, p.M - m0), ncols = min(BN, p.N - n0);  // valid part of the output tile
    uint32_t cols = 32;
    while (cols < static_cast<uint32_t>(BN)) cols <<= 1;

    if (tid == 0) {
        mbar_init(smem_u32(bar), 1);
        mbar_init(smem_u32(bar + 1), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(cols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    // weight gradient with bias partials: B gets a virtual row N of ones, so column N
    // of the product holds the column sums of A^T (the bias gradient)
    const bool with_bias = MODE == PB_TRAIN_DW && p.col_part != nullptr;
    const bool tma = p.tma_a || p.tma_b;
    if (tma) {
        __syncthreads();  // the barrier's initialisation is visible before the copies arrive on it
        if (tid == 0) {
            mbar_expect_tx(smem_u32(bar + 1),
                           (p.tma_a ? kRows * KC * 2u : 0u) + (p.tma_b ? static_cast<uint32_t>(BN) * KC * 2u : 0u));
            if (p.tma_a) tma_load_tile(smem_u32(As), &map_a, k0, m0, smem_u32(bar + 1));
            if (p.tma_b) tma_load_tile(smem_u32(Bs), &map_b, k0, n0, smem_u32(bar + 1));
        }
    }
    if (!p.tma_a) {
        if constexpr (AK)
            stage_kcontig(As, p.A, p.sam, m0, kRows, p.M, k0, KC, kend, -1);
        else
            stage_rowcontig(As, p.A, p.sam, p.sak, m0, kRows, p.M, k0, KC, kend, -1);
    }
    if (!p.tma_b) {
        if constexpr (BK)
            stage_kcontig(Bs, p.B, p.sbn, n0, BN, p.N, k0, KC, kend, with_bias ? p.N : -1);
        else
            stage_rowcontig(Bs, p.B, p.sbn, p.sbk, n0, BN, p.N, k0, KC, kend, with_bias ? p.N : -1);
    }
    cp_async_wait_all();
    bool staged = true;
    if (tma) {
        staged = !__syncthreads_or(!mbar_wait(smem_u32(bar + 1), 0));
        if (p.tma_b && with_bias && p.N - n0 >= 0 && p.N - n0 < BN) ones_row(Bs, p.N - n0, KC, k0, kend);
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    if (tid == 0 && staged) {
        const uint32_t sbo_a = static_cast<uint32_t>(KC >> 3) << 7;
        const uint32_t idesc = instr_desc(kRows, BN);
        for (int kk = 0; kk < (KC >> 4); ++kk)
            mma_bf16(tmem, smem_desc(smem_u32(As) + kk * 256u, 128u, sbo_a),
                     smem_desc(smem_u32(Bs) + kk * 256u, 128u, sbo_a), idesc, kk > 0 ? 1u : 0u);
        mma_commit(smem_u32(bar));
    }
    const int fp = (BN + 4) * 4;  // pitch of the z_in tile (bytes)
    if constexpr (MODE == PB_TRAIN_DX) {
        // the pre-activations of this tile, into their own region while the MMAs run
        uint8_t* zt = smem + p.zin_off;
        const int per_row = BN / 4;
        for (int idx = tid; idx < kRows * per_row; idx += kThreads) {
            const int r = idx / per_row, c = (idx - r * per_row) * 4;
            float* d = reinterpret_cast<float*>(zt + r * fp) + c;
            const float* src = p.z_in + static_cast<int64_t>(m0 + r) * p.ldz + n0 + c;
            if (r < rows && c + 4 <= ncols && aligned16(src)) {
                cp_async16(smem_u32(d), src);
            } else {
                for (int j = 0; j < 4; ++j) d[j] = (r < rows && c + j < ncols) ? src[j] : 0.f;
            }
        }
        cp_async_wait_all();
    }
    const bool ok = staged && !__syncthreads_or(!mbar_wait(smem_u32(bar), 0));
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (ok) {
        const int quarter = warp & 3, half = warp >> 2;
        const int r = quarter * 32 + lane;  // this thread's row of the tile (its TMEM lane)
        const int m = m0 + r;
        const bool row_ok = r < rows;
        for (int c0 = half * 32; c0 < BN; c0 += 64) {
            uint32_t raw[32];
            tmem_ld32(tmem + (static_cast<uint32_t>(quarter * 32) << 16) + static_cast<uint32_t>(c0), raw);
            float v[32];
#pragma unroll
            for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(raw[j]);
            if constexpr (MODE == PB_TRAIN_FWD_GELU) {
                // z (FP32) and GELU(z) (BF16) from registers, 16-byte stores along the
                // row; the transposed copy column by column (a column's 32 rows are 64
                // contiguous bytes)
                if (row_ok) {
#pragma unroll
                    for (int g = 0; g < 32; g += 8) {
                        if (c0 + g >= ncols) break;
                        const int n = n0 + c0 + g;
                        const int64_t o = static_cast<int64_t>(m) * p.ldc + n;
                        float z[8];
                        __align__(16) __nv_bfloat16 h[8];
#pragma unroll
                        for (int j = 0; j < 8; ++j) {
                            z[j] = v[g + j] + (c0 + g + j < ncols ? __ldg(p.bias + n + j) : 0.f);
                            h[j] = __float2bfloat16(gelu(z[j]));
                        }
                        if (c0 + g + 8 <= ncols && (o & 7) == 0 && aligned16(p.out_bf16) &&
                            (!p.z_pre || aligned16(p.z_pre))) {
                            if (p.z_pre) {
                                reinterpret_cast<float4*>(p.z_pre + o)[0] = make_float4(z[0], z[1], z[2], z[3]);
                                reinterpret_cast<float4*>(p.z_pre + o)[1] = make_float4(z[4], z[5], z[6], z[7]);
                            }
                            *reinterpret_cast<uint4*>(p.out_bf16 + o) = *reinterpret_cast<const uint4*>(h);
                        } else {
#pragma unroll
                            for (int j = 0; j < 8; ++j)
                                if (c0 + g + j < ncols) {
                                    if (p.z_pre) p.z_pre[o + j] = z[j];
                                    p.out_bf16[o + j] = h[j];
                                }
                        }
                        if (p.out_t) {
#pragma unroll
                            for (int j = 0; j < 8; ++j)
                                if (c0 + g + j < ncols) p.out_t[static_cast<int64_t>(n + j) * p.ldt + m] = h[j];
                        }
                    }
                }
            } else if constexpr (MODE == PB_TRAIN_FWD_LINEAR) {
                if (row_ok) {
#pragma unroll
                    for (int j = 0; j < 32; ++j) {
                        const int n = n0 + c0 + j;
                        if (c0 + j < ncols)
                            p.out_f32[static_cast<int64_t>(m) * p.ldc + n] = v[j] + (p.bias ? __ldg(p.bias + n) : 0.f);
                    }
                }
            } else if constexpr (MODE == PB_TRAIN_DX) {
                // pre-activations from the tile loaded during the MMAs
                const float* zt = reinterpret_cast<const float*>(smem + p.zin_off + r * fp) + c0;
#pragma unroll
                for (int g = 0; g < 32; g += 8) {
                    if (c0 + g >= BN) {  // past the tile: zero for the column sums
#pragma unroll
                        for (int j = 0; j < 8; ++j) v[g + j] = 0.f;
                        continue;
                    }
                    const int n = n0 + c0 + g;
                    const int64_t o = static_cast<int64_t>(m) * p.ldc + n;
                    const float4 z0 = reinterpret_cast<const float4*>(zt + g)[0];
                    const float4 z1 = reinterpret_cast<const float4*>(zt + g)[1];
                    const float z[8] = {z0.x, z0.y, z0.z, z0.w, z1.x, z1.y, z1.z, z1.w};
                    __align__(16) __nv_bfloat16 h[8];
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        const bool ok_j = row_ok && c0 + g + j < ncols;
                        v[g + j] = ok_j ? v[g + j] * gelu_grad(z[j]) : 0.f;
                        h[j] = __float2bfloat16(v[g + j]);
                    }
                    if (row_ok) {
                        if (c0 + g + 8 <= ncols && (o & 7) == 0 && aligned16(p.out_bf16)) {
                            *reinterpret_cast<uint4*>(p.out_bf16 + o) = *reinterpret_cast<const uint4*>(h);
                        } else {
#pragma unroll
                            for (int j = 0; j < 8; ++j)
                                if (c0 + g + j < ncols) p.out_bf16[o + j] = h[j];
                        }
                        if (p.out_t) {
#pragma unroll
                            for (int j = 0; j < 8; ++j)
                                if (c0 + g + j < ncols) p.out_t[static_cast<int64_t>(n + j) * p.ldt + m] = h[j];
                        }
                    }
                }
                if (p.col_part) {
                    const float cs = warp_column_sums(v, lane);  // lane j: column c0 + j over this warp's rows
                    if (c0 + lane < ncols)
                        p.col_part[static_cast<int64_t>(blockIdx.x * 4 + quarter) * p.ldp + n0 + c0 + lane] = cs;
                }
            } else {  // PB_TRAIN_DW: the split-K partial (and the bias partial from the ones column)
                if (row_ok) {
                    float* o = p.out_f32 + static_cast<int64_t>(blockIdx.z) * p.M * p.ldc + static_cast<int64_t>(m) * p.ldc + n0;
#pragma unroll
                    for (int g = 0; g < 32; g += 8) {
                        if (c0 + g >= BN) break;
                        if (c0 + g + 8 <= ncols && aligned16(o + c0 + g)) {
                            reinterpret_cast<float4*>(o + c0 + g)[0] = make_float4(v[g], v[g + 1], v[g + 2], v[g + 3]);
                            reinterpret_cast<float4*>(o + c0 + g)[1] =
                                make_float4(v[g + 4], v[g + 5], v[g + 6], v[g + 7]);
                        } else {
#pragma unroll
                            for (int j = 0; j < 8; ++j)
                                if (c0 + g + j < ncols) o[c0 + g + j] = v[g + j];
                        }
                    }
                    const int jb = p.N - n0 - c0;  // the ones column, if it falls in this chunk
                    if (with_bias && jb >= 0 && jb < 32 && c0 + jb < BN) {
#pragma unroll
                        for (int j = 0; j < 32; ++j)
                            if (j == jb) p.col_part[static_cast<int64_t>(blockIdx.z) * p.ldp + m] = v[j];
                    }
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (!ok && tid == 0 && p.error) atomicExch(p.error, 1);
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(cols) : "memory");
}

// Softmax cross-entropy of logits (M x C, row stride ldl) against labels:
// dz = (p - onehot(y)) * scale in BF16 (row stride ldd), loss and correct counts
// accumulated, and per-block column sums of dz (the last layer's bias gradient)
// into part[blockIdx.x * C + c].
constexpr int kXentThreads = 256;
constexpr int kMaxClasses = 32;
__global__ void __launch_bounds__(kXentThreads) k_xent(const float* __restrict__ logits, int64_t ldl,
                                                      const int32_t* __restrict__ y, int M, int C, float scale,
                                                      __nv_bfloat16* __restrict__ dz, int64_t ldd,
                                                      __nv_bfloat16* __restrict__ dz_t, int64_t ldt,
                                                      float* __restrict__ part, float* __restrict__ loss_sum,
                                                      int32_t* __restrict__ correct)
{
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    float my_loss = 0.f;
    int my_hit = 0;
    float g[kMaxClasses];
    for (int c = 0; c < kMaxClasses; ++c) g[c] = 0.f;
    if (m < M) {
        const float* l = logits + static_cast<int64_t>(m) * ldl;
        float mx = -CUDART_INF_F;
        int arg = 0;
        for (int c = 0; c < C; ++c)
            if (l[c] > mx) {
                mx = l[c];
                arg = c;
            }
        float s = 0.f;
        for (int c = 0; c < C; ++c) s += __expf(l[c] - mx);
        const int yc = y[m];
        const float inv = 1.f / s;
        for (int c = 0; c < C; ++c) {
            const float pc = __expf(l[c] - mx) * inv;
            g[c] = (pc - (c == yc ? 1.f : 0.f)) * scale;
            const __nv_bfloat16 h = __float2bfloat16(g[c]);
            dz[static_cast<int64_t>(m) * ldd + c] = h;
            if (dz_t) dz_t[static_cast<int64_t>(c) * ldt + m] = h;
        }
        if (yc >= 0 && yc < C) {
            my_loss = -(l[yc] - mx - __logf(s));
            my_hit = arg == yc ? 1 : 0;
        }
    }
    // loss and hits: warp sums, then one atomic per block
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) {
        my_loss += __shfl_xor_sync(0xffffffffu, my_loss, o);
        my_hit += __shfl_xor_sync(0xffffffffu, my_hit, o);
    }
    // per-warp sums in a fixed order, then warps in order: deterministic
    for (int c = 0; c < C; ++c) {
        float v = g[c];
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        g[c] = v;
    }
    __shared__ float wsum[kXentThreads / 32][kMaxClasses];
    __shared__ float wloss[kXentThreads / 32];
    __shared__ int whit[kXentThreads / 32];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        for (int c = 0; c < C; ++c) wsum[warp][c] = g[c];
        wloss[warp] = my_loss;
        whit[warp] = my_hit;
    }
    __syncthreads();
    if (part && threadIdx.x < C) {
        float s = 0.f;
        for (int w = 0; w < kXentThreads / 32; ++w) s += wsum[w][threadIdx.x];
        part[static_cast<int64_t>(blockIdx.x) * C + threadIdx.x] = s;
    }
    if (threadIdx.x == 0) {
        float ls = 0.f;
        int hs = 0;
        for (int w = 0; w < kXentThreads / 32; ++w) {
            ls += wloss[w];
            hs += whit[w];
        }
        if (loss_sum) atomicAdd(loss_sum, ls);
        if (correct && hs) atomicAdd(correct, hs);
    }
}

struct AdamSeg {
    float* w;               // FP32 master weights (n = rows x cols, row-major)
    __nv_bfloat16* wb;      // BF16 copy (n), optional
    __nv_bfloat16* wbt;     // BF16 copy transposed (cols x rows), optional
    int64_t cols;
    float* m1;
    float* m2;
    const float* gpart;     // gradient partials: part p of element i at gpart[p * pstride + i]
    int64_t n, pstride;
    int nparts;
    float wd;
};

struct AdamArgs {
    AdamSeg seg[kMaxSeg];
    int64_t off[kMaxSeg + 1];  // prefix offsets of the segments
    int nseg;
    float lr, b1, b2, eps, bc1, bc2;
};

__global__ void k_adamw_multi(const AdamArgs a)
{
    const int64_t total = a.off[a.nseg];
    for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < total;
         e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        int s = 0;
        while (s + 1 < a.nseg && e >= a.off[s + 1]) ++s;
        const AdamSeg& g = a.seg[s];
        const int64_t i = e - a.off[s];
        // partials in a fixed order, four loads in flight
        float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f;
        int q = 0;
        for (; q + 4 <= g.nparts; q += 4) {
            a0 += g.gpart[(q + 0) * g.pstride + i];
            a1 += g.gpart[(q + 1) * g.pstride + i];
            a2 += g.gpart[(q + 2) * g.pstride + i];
            a3 += g.gpart[(q + 3) * g.pstride + i];
        }
        for (; q < g.nparts; ++q) a0 += g.gpart[q * g.pstride + i];
        const float gi = (a0 + a1) + (a2 + a3);
        const float m1 = a.b1 * g.m1[i] + (1.f - a.b1) * gi;
        const float m2 = a.b2 * g.m2[i] + (1.f - a.b2) * gi * gi;
        g.m1[i] = m1;
        g.m2[i] = m2;
        float w = g.w[i] * (1.f - a.lr * g.wd);
        w -= a.lr * (m1 / a.bc1) / (sqrtf(m2 / a.bc2) + a.eps);
        g.w[i] = w;
        const __nv_bfloat16 h = __float2bfloat16(w);
        if (g.wb) g.wb[i] = h;
        if (g.wbt) {
            const int64_t r = i / g.cols, c = i - r * g.cols;
            g.wbt[c * (g.n / g.cols) + r] = h;
        }
    }
}

// out[k] = x[idx[k]] (rows of `width` BF16), y_out[k] = y[idx[k]]
__global__ void k_gather_train(const __nv_bfloat16* __restrict__ x, int width, const int32_t* __restrict__ y,
                               const int32_t* __restrict__ idx, int64_t n, __nv_bfloat16* __restrict__ out,
                               __nv_bfloat16* __restrict__ out_t, int32_t* __restrict__ y_out)
{
    for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < n * width;
         e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t k = e / width;
        const int c = static_cast<int>(e - k * width);
        const int64_t src = idx[k];
        const __nv_bfloat16 v = x[src * width + c];
        out[e] = v;
        if (out_t) out_t[c * n + k] = v;
        if (c == 0 && y_out) y_out[k] = y[src];
    }
}

using GemmFn = void (*)(GemmTcArgs, CUtensorMap, CUtensorMap);

template <int MODE>
constexpr GemmFn gemm_of(bool ak, bool bk)
{
    return ak ? (bk ? k_gemm_tc<MODE, true, true> : k_gemm_tc<MODE, true, false>)
              : (bk ? k_gemm_tc<MODE, false, true> : k_gemm_tc<MODE, false, false>);
}

GemmFn gemm_kernel(int mode, bool ak, bool bk)
{
    switch (mode) {
        case PB_TRAIN_FWD_GELU: return gemm_of<PB_TRAIN_FWD_GELU>(ak, bk);
        case PB_TRAIN_FWD_LINEAR: return gemm_of<PB_TRAIN_FWD_LINEAR>(ak, bk);
        case PB_TRAIN_DX: return gemm_of<PB_TRAIN_DX>(ak, bk);
        default: return gemm_of<PB_TRAIN_DW>(ak, bk);
    }
}

// the GEMMs' dynamic shared memory limit, raised once per device for every
// instance (outside any stream capture that follows)
cudaError_t ensure_gemm_smem()
{
    constexpr int kDevs = 64;
    static std::atomic<int> done[kDevs];
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev >= 0 && dev < kDevs && done[dev].load(std::memory_order_acquire)) return cudaSuccess;
    for (int mode = 0; mode < 4 && e == cudaSuccess; ++mode)
        for (int c = 0; c < 4 && e == cudaSuccess; ++c)
            e = cudaFuncSetAttribute(gemm_kernel(mode, c & 1, c & 2), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     kMaxSmem);
    if (e == cudaSuccess && dev >= 0 && dev < kDevs) done[dev].store(1, std::memory_order_release);
    return e;
}

// cuTensorMapEncodeTiled through the runtime's driver entry points (the library
// does not link libcuda); nullptr if unavailable (the copies then use cp.async)
using FnEncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
// PB_TRAIN_NO_TMA=1 in the environment keeps every copy on cp.async (a comparison switch)
bool no_tma()
{
    static const bool off = [] {
        const char* v = getenv("PB_TRAIN_NO_TMA");
        return v && v[0] == '1';
    }();
    return off;
}

FnEncodeTiled encode_tiled()
{
    static FnEncodeTiled fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* q = nullptr;
        cudaDriverEntryPointQueryResult r;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &q, cudaEnableDefault, &r) == cudaSuccess &&
            r == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<FnEncodeTiled>(q);
    });
    return fn;
}

// The 4-D tensor map of a K-contiguous operand X (rows x K, row pitch sr
// elements) whose (8 k x 8 rows x kc/8 x rows_box/8) box is a run of core
// matrices; false (no map) unless rows and K are multiples of 8 and the rows
// 16-byte aligned.
bool operand_map(CUtensorMap* map, const void* X, int64_t sr, int rows, int K, int kc, int rows_box)
{
    const FnEncodeTiled enc = encode_tiled();
    if (!enc || rows % 8 || K % 8 || (sr * 2) % 16 || reinterpret_cast<uintptr_t>(X) % 16 || rows_box % 8 ||
        rows_box > 256 * 8 || kc > 256 * 8)
        return false;
    const cuuint64_t dims[4] = {8, 8, static_cast<cuuint64_t>(K / 8), static_cast<cuuint64_t>(rows / 8)};
    const cuuint64_t strides[3] = {static_cast<cuuint64_t>(sr * 2), 16, static_cast<cuuint64_t>(sr * 2 * 8)};
    const cuuint32_t box[4] = {8, 8, static_cast<cuuint32_t>(kc / 8), static_cast<cuuint32_t>(rows_box / 8)};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    return enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void*>(X), dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

int grid_cap(int64_t work, int block)
{
    int64_t g = (work + block - 1) / block;
    if (g > 148 * 16) g = 148 * 16;
    return static_cast<int>(g < 1 ? 1 : g);
}

}  // namespace

extern "C" {

int pb_train_gemm(const void* A, int64_t sam, int64_t sak, const void* B, int64_t sbn, int64_t sbk, int32_t M,
                  int32_t N, int32_t K, int32_t mode, int32_t kc, int32_t bn, const float* bias, const float* z_in,
                  int64_t ldz, float* out_f32, void* out_bf16, void* out_t, float* z_pre, float* col_part,
                  int64_t ldc, int64_t ldt, int64_t ldp, int32_t* error_flag, void* stream)
{
    if (!A || !B || M < 0 || N < 0 || K < 1) return PB_EINVAL;
    if (kc < 16 || kc > kMaxKc || kc % 16 || bn < 16 || bn > kMaxBn || bn % 16) return PB_EINVAL;
    // each operand is contiguous along K or along its rows (16-byte reads of 8 elements)
    if ((sak != 1 && sam != 1) || (sbk != 1 && sbn != 1)) return PB_EINVAL;
    if (ldc < N || (out_t && ldt < M)) return PB_EINVAL;
    switch (mode) {
        case PB_TRAIN_FWD_GELU:
            if (!bias || !out_bf16 || kc < K) return PB_EINVAL;
            break;
        case PB_TRAIN_FWD_LINEAR:
            if (!out_f32 || kc < K) return PB_EINVAL;
            break;
        case PB_TRAIN_DX:
            if (!z_in || !out_bf16 || ldz < N || kc < K || (col_part && ldp < N)) return PB_EINVAL;
            break;
        case PB_TRAIN_DW:
            if (!out_f32 || (col_part && ldp < M)) return PB_EINVAL;
            break;
        default: return PB_EINVAL;
    }
    if (M == 0 || N == 0) return PB_SUCCESS;
    GemmTcArgs p{};
    p.A = static_cast<const __nv_bfloat16*>(A);
    p.B = static_cast<const __nv_bfloat16*>(B);
    p.sam = sam;
    p.sak = sak;
    p.sbn = sbn;
    p.sbk = sbk;
    p.M = M;
    p.N = N;
    p.K = K;
    p.kc = kc;
    p.bn = bn;
    p.mode = mode;
    p.bias = bias;
    p.z_in = z_in;
    p.ldz = ldz;
    p.out_f32 = out_f32;
    p.out_bf16 = static_cast<__nv_bfloat16*>(out_bf16);
    p.out_t = static_cast<__nv_bfloat16*>(out_t);
    p.z_pre = z_pre;
    p.col_part = col_part;
    p.ldc = ldc;
    p.ldt = ldt;
    p.ldp = ldp;
    p.error = error_flag;
    const int n_cols = N + ((mode == PB_TRAIN_DW && col_part) ? 1 : 0);  // + the ones column
    const dim3 grid((M + kRows - 1) / kRows, (n_cols + bn - 1) / bn, (K + kc - 1) / kc);
    if (grid.y > 65535 || grid.z > 65535) return PB_EINVAL;
    int smem = 0;
    smem_plan(mode, kc, bn, &p.zin_off, &p.bar_off, &smem);
    if (smem > kMaxSmem) return PB_EINVAL;  // e.g. the input gradient with bn > 128
    if (ensure_gemm_smem() != cudaSuccess) return PB_ECUDA;
    CUtensorMap map_a{}, map_b{};
    if (!no_tma()) {
        p.tma_a = sak == 1 && operand_map(&map_a, A, sam, M, K, kc, kRows) ? 1 : 0;
        p.tma_b = sbk == 1 && operand_map(&map_b, B, sbn, N, K, kc, bn) ? 1 : 0;
    }
    gemm_kernel(mode, sak == 1, sbk == 1)<<<grid, kThreads, smem, static_cast<cudaStream_t>(stream)>>>(p, map_a,
                                                                                                      map_b);
    return cudaGetLastError() == cudaSuccess ? PB_SUCCESS : PB_ECUDA;
}

int pb_train_xent(const float* logits, int64_t ldl, const int32_t* labels, int32_t M, int32_t C, float scale,
                  void* dz_bf16, int64_t ldd, void* dz_t, int64_t ldt, float* bias_part, float* loss_sum,
                  int32_t* correct, void* stream)
{
    if (!logits || !labels || !dz_bf16 || M < 0 || C < 1 || C > kMaxClasses || ldl < C || ldd < C ||
        (dz_t && ldt < M))
        return PB_EINVAL;
    if (M == 0) return PB_SUCCESS;
    k_xent<<<(M + kXentThreads - 1) / kXentThreads, kXentThreads, 0, static_cast<cudaStream_t>(stream)>>>(
        logits, ldl, labels, M, C, scale, static_cast<__nv_bfloat16*>(dz_bf16), ldd,
        static_cast<__nv_bfloat16*>(dz_t), ldt, bias_part, loss_sum, correct);
    return cudaGetLastError() == cudaSuccess ? PB_SUCCESS : PB_ECUDA;
}

int pb_train_xent_parts(int32_t M) { return M < 0 ? -1 : (M + kXentThreads - 1) / kXentThreads; }

int pb_train_adamw(int32_t n_tensors, float* const* w, void* const* w_bf16, void* const* w_bf16_t,
                   const int64_t* cols, float* const* m1, float* const* m2, const float* const* grad_parts,
                   const int64_t* n, const int64_t* part_stride, const int32_t* n_parts, const float* weight_decay,
                   float lr, float beta1, float beta2, float eps, int32_t step, void* stream)
{
    if (n_tensors < 1 || n_tensors > kMaxSeg || !w || !m1 || !m2 || !grad_parts || !n || !part_stride || !n_parts ||
        !weight_decay || step < 1)
        return PB_EINVAL;
    AdamArgs a{};
    a.nseg = n_tensors;
    a.off[0] = 0;
    for (int s = 0; s < n_tensors; ++s) {
        if (!w[s] || !m1[s] || !m2[s] || !grad_parts[s] || n[s] < 0 || n_parts[s] < 1 || part_stride[s] < n[s])
            return PB_EINVAL;
        void* wt = w_bf16_t ? w_bf16_t[s] : nullptr;
        const int64_t nc = cols ? cols[s] : 1;
        if (wt && (nc < 1 || n[s] % nc)) return PB_EINVAL;
        a.seg[s] = AdamSeg{w[s], w_bf16 ? static_cast<__nv_bfloat16*>(w_bf16[s]) : nullptr,
                           static_cast<__nv_bfloat16*>(wt), nc, m1[s], m2[s], grad_parts[s], n[s], part_stride[s],
                           n_parts[s], weight_decay[s]};
        a.off[s + 1] = a.off[s] + n[s];
    }
    a.lr = lr;
    a.b1 = beta1;
    a.b2 = beta2;
    a.eps = eps;
    a.bc1 = 1.f - powf(beta1, static_cast<float>(step));
    a.bc2 = 1.f - powf(beta2, static_cast<float>(step));
    if (a.off[n_tensors] == 0) return PB_SUCCESS;
    k_adamw_multi<<<grid_cap(a.off[n_tensors], 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(a);
    return cudaGetLastError() == cudaSuccess ? PB_SUCCESS : PB_ECUDA;
}

int pb_train_gather(const void* x_bf16, int32_t width, const int32_t* labels, const int32_t* idx, int64_t n,
                    void* out_bf16, void* out_t, int32_t* labels_out, void* stream)
{
    if (!x_bf16 || !idx || !out_bf16 || width < 1 || n < 0 || (labels_out && !labels)) return PB_EINVAL;
    if (n == 0) return PB_SUCCESS;
    k_gather_train<<<grid_cap(n * width, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<const __nv_bfloat16*>(x_bf16), width, labels, idx, n, static_cast<__nv_bfloat16*>(out_bf16),
        static_cast<__nv_bfloat16*>(out_t), labels_out);
    return cudaGetLastError() == cudaSuccess ? PB_SUCCESS : PB_ECUDA;
}

}  // extern "C"
