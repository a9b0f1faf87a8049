// Surrogate inference on the 5th-generation tensor cores.
//
// One CTA evaluates the whole MLP for a tile of 128 rows: every layer is a
// tcgen05.mma (M = 128, N <= 256, K <= 256, BF16 x BF16 -> FP32) whose
// accumulator lives in tensor memory; the epilogue reads it back with
// tcgen05.ld, adds the bias, applies GELU and writes the BF16 activations into
// shared memory as the next layer's A operand, so activations never leave the
// SM.  Each layer's weights (pre-packed on the host in the operand layout) are
// streamed from global memory / L2 into shared memory by bulk copies completing
// on an mbarrier; the copy for layer l+1 starts as soon as the MMAs of layer l
// have finished reading, overlapping the epilogue.  One thread issues the MMAs;
// 16 warps run the epilogue: warp w reads TMEM lanes 32 (w % 4) .. + 31 (the
// lane quarter a warp may access) and every fourth 32-column chunk starting at
// chunk w / 4, so the bias + GELU work is spread over 512 threads.
//
// Operand layout (K-major, no swizzle): 8-row x 16-byte core matrices, core
// (row/8, k/8) at ((row/8) * (K/8) + k/8) * 128 bytes; in the shared-memory
// descriptor the leading byte offset is the K-direction core stride (128 B) and
// the stride byte offset the 8-row-group stride ((K/8) * 128 B).
//
// Every mbarrier wait is bounded: on a timeout the CTA sets the error flag,
// frees its tensor memory and exits.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "pb_gelu.cuh"
#include "pybasin_b200.h"

namespace {

constexpr int kRows = 128;      // rows per CTA = MMA M = TMEM lanes used
constexpr int kMaxDim = 256;    // largest K and N of a layer
constexpr int kMaxLayers = 8;
constexpr int kThreads = 512;
constexpr int kColGroups = kThreads / 128;  // warps sharing one TMEM lane quarter
constexpr uint32_t kTmemCols = 256;
constexpr int kABytes = kRows * kMaxDim * 2;      // activations, 64 KB
constexpr int kBBytes = kMaxDim * kMaxDim * 2;    // one layer's weights, 128 KB
constexpr int kSmemBytes = kABytes + kBBytes + 64;
constexpr long long kWaitPolls = 1ll << 22;       // polls of an mbarrier before giving up
constexpr uint32_t kCopyChunk = 32768;            // bytes per bulk copy

struct MlpTcArgs {
    const __nv_bfloat16* x;  // (n, d_in) row-major
    int64_t n;
    int d_in;
    int n_layers;
    int n_classes;
    int _pad;
    const uint8_t* w[kMaxLayers];  // packed weights of layer l: n_pad x k_pad BF16 in the operand layout
    const float* b[kMaxLayers];    // bias of layer l (n_real entries)
    int n_pad[kMaxLayers], k_pad[kMaxLayers], n_real[kMaxLayers];
    float* logits;  // (n, n_classes)
    int* error;     // set to 1 when a wait gave up
};

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint32_t core_offset(int row, int k, int K)
{
    return ((static_cast<uint32_t>(row >> 3) * static_cast<uint32_t>(K >> 3) + static_cast<uint32_t>(k >> 3)) << 7) +
           (static_cast<uint32_t>(row & 7) << 4) + (static_cast<uint32_t>(k & 7) << 1);
}

// shared-memory matrix descriptor: start address, leading / stride byte offsets
// (16-byte units), descriptor version 1, base offset 0, no swizzle
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    return static_cast<uint64_t>((addr >> 4) & 0x3FFFu) | (static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16) |
           (static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both K-major
__device__ __forceinline__ uint32_t instr_desc(int M, int N)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(N >> 3) << 17) |
           (static_cast<uint32_t>(M >> 4) << 24);
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
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

// true once the phase of the given parity completed; false after kWaitPolls polls
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity)
{
    for (long long i = 0; i < kWaitPolls; ++i)
        if (mbar_try(bar, parity)) return true;
    return false;
}

__device__ __forceinline__ void bulk_copy(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

// weights of one layer into the B buffer (issued by one thread)
__device__ __forceinline__ void load_weights(const MlpTcArgs& p, int l, uint32_t b_smem, uint32_t bar)
{
    const uint32_t bytes = static_cast<uint32_t>(p.n_pad[l]) * static_cast<uint32_t>(p.k_pad[l]) * 2u;
    mbar_expect_tx(bar, bytes);
    for (uint32_t off = 0; off < bytes; off += kCopyChunk) {
        const uint32_t len = bytes - off < kCopyChunk ? bytes - off : kCopyChunk;
        bulk_copy(b_smem + off, p.w[l] + off, len, bar);
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

// 32 consecutive FP32 columns of this thread's TMEM lane
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

using pb::gelu;

__global__ void __launch_bounds__(kThreads, 1) k_mlp_infer_tc(const MlpTcArgs p)
{
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t* As = smem;
    uint8_t* Bs = smem + kABytes;
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kABytes + kBBytes);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int quarter = warp & 3, cgroup = warp >> 2;
    const int trow = quarter * 32 + lane;  // this thread's row of the tile (its TMEM lane)
    const uint32_t bar_w = smem_u32(&bars[0]), bar_m = smem_u32(&bars[1]);
    const uint32_t a_smem = smem_u32(As), b_smem = smem_u32(Bs);
    const int64_t row0 = static_cast<int64_t>(blockIdx.x) * kRows;
    const int64_t row = row0 + trow;

    if (tid == 0) {
        mbar_init(bar_w, 1);
        mbar_init(bar_m, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    if (tid == 0) load_weights(p, 0, b_smem, bar_w);
    {  // layer-0 operand, 8 columns of one row per step; zero beyond d_in and beyond n
        const int K = p.k_pad[0];
        for (int idx = tid; idx < kRows * (K >> 3); idx += kThreads) {
            const int r = idx & (kRows - 1), k = (idx / kRows) * 8;
            const int64_t gr = row0 + r;
            __align__(16) __nv_bfloat16 h[8];
#pragma unroll
            for (int j = 0; j < 8; ++j)
                h[j] = (gr < p.n && k + j < p.d_in) ? p.x[gr * p.d_in + k + j] : __float2bfloat16(0.f);
            *reinterpret_cast<uint4*>(As + core_offset(r, k, K)) = *reinterpret_cast<const uint4*>(h);
        }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();

    uint32_t ph_w = 0, ph_m = 0;
    bool ok = true;
    for (int l = 0; l < p.n_layers && ok; ++l) {
        const int N = p.n_pad[l], K = p.k_pad[l];
        ok = !__syncthreads_or(!mbar_wait(bar_w, ph_w));
        ph_w ^= 1u;
        if (!ok) break;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (tid == 0) {
            const uint32_t sbo = static_cast<uint32_t>(K >> 3) << 7;
            const uint32_t idesc = instr_desc(kRows, N);
            for (int kk = 0; kk < (K >> 4); ++kk)
                mma_bf16(tmem, smem_desc(a_smem + kk * 256u, 128u, sbo), smem_desc(b_smem + kk * 256u, 128u, sbo),
                         idesc, kk > 0 ? 1u : 0u);
            mma_commit(bar_m);
        }
        ok = !__syncthreads_or(!mbar_wait(bar_m, ph_m));
        ph_m ^= 1u;
        if (!ok) break;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (tid == 0 && l + 1 < p.n_layers) load_weights(p, l + 1, b_smem, bar_w);  // B is free again
        const bool last = l + 1 == p.n_layers;
        const float* bias = p.b[l];
        const int nr = p.n_real[l];
        for (int c0 = cgroup * 32; c0 < N; c0 += 32 * kColGroups) {
            uint32_t v[32];
            tmem_ld32(tmem + (static_cast<uint32_t>(quarter * 32) << 16) + static_cast<uint32_t>(c0), v);
            if (!last) {
                for (int g = 0; g < 32 && c0 + g < N; g += 8) {
                    __align__(16) __nv_bfloat16 h[8];
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        const int c = c0 + g + j;
                        const float z = __uint_as_float(v[g + j]) + (c < nr ? __ldg(bias + c) : 0.f);
                        h[j] = __float2bfloat16(c < nr ? gelu(z) : 0.f);
                    }
                    *reinterpret_cast<uint4*>(As + core_offset(trow, c0 + g, N)) = *reinterpret_cast<const uint4*>(h);
                }
            } else if (row < p.n) {
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    const int c = c0 + j;
                    if (c < p.n_classes) p.logits[row * p.n_classes + c] = __uint_as_float(v[j]) + __ldg(bias + c);
                }
            }
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
    }
    if (!ok && tid == 0 && p.error) atomicExch(p.error, 1);
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
}

}  // namespace

extern "C" int pb_mlp_infer_tc(const void* x_bf16, int64_t n, int32_t d_in, int32_t n_layers,
                               const void* const* w_packed, const float* const* bias, const int32_t* n_pad,
                               const int32_t* k_pad, const int32_t* n_real, float* logits, int32_t n_classes,
                               int32_t* error_flag, void* stream)
{
    if (n < 0 || n_layers < 1 || n_layers > kMaxLayers || d_in < 1) return PB_EINVAL;
    if (n == 0) return PB_SUCCESS;
    if (!x_bf16 || !w_packed || !bias || !n_pad || !k_pad || !n_real || !logits) return PB_EINVAL;
    MlpTcArgs p{};
    p.x = static_cast<const __nv_bfloat16*>(x_bf16);
    p.n = n;
    p.d_in = d_in;
    p.n_layers = n_layers;
    p.n_classes = n_classes;
    p.logits = logits;
    p.error = error_flag;
    if (k_pad[0] < d_in) return PB_EINVAL;
    for (int l = 0; l < n_layers; ++l) {
        const int N = n_pad[l], K = k_pad[l];
        if (N < 16 || N > kMaxDim || N % 16 || K < 16 || K > kMaxDim || K % 16) return PB_EINVAL;
        if (n_real[l] < 1 || n_real[l] > N || !w_packed[l] || !bias[l]) return PB_EINVAL;
        if (reinterpret_cast<uintptr_t>(w_packed[l]) % 16) return PB_EINVAL;  // bulk copies need 16-byte alignment
        if (l > 0 && K != n_pad[l - 1]) return PB_EINVAL;
        p.w[l] = static_cast<const uint8_t*>(w_packed[l]);
        p.b[l] = bias[l];
        p.n_pad[l] = N;
        p.k_pad[l] = K;
        p.n_real[l] = n_real[l];
    }
    if (n_classes < 1 || n_classes > n_real[n_layers - 1]) return PB_EINVAL;
    cudaError_t e = cudaFuncSetAttribute(k_mlp_infer_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes);
    if (e != cudaSuccess) return PB_ECUDA;
    const int64_t grid = (n + kRows - 1) / kRows;
    if (grid > 0x7fffffffLL) return PB_EINVAL;
    k_mlp_infer_tc<<<static_cast<unsigned>(grid), kThreads, kSmemBytes, static_cast<cudaStream_t>(stream)>>>(p);
    return cudaGetLastError() == cudaSuccess ? PB_SUCCESS : PB_ECUDA;
}
