// Fused surrogate training step on the 5th-generation tensor cores.
//
// One minibatch step of the MLP (layers dims[0] -> ... -> dims[L], GELU between,
// softmax cross-entropy on the logits, AdamW) is two launches:
//
//   k_train_fb   one CTA per 128-row tile of the minibatch runs the whole layer
//                chain of its rows: it gathers its input rows, runs every layer's
//                forward GEMM, the cross entropy, and every layer's input-gradient
//                GEMM, keeping activations and gradients in shared memory.  For
//                the weight gradients it leaves each layer's input X_l and output
//                gradient dZ_l of its rows in global scratch (as images of the
//                shared-memory operand layout), and GELU'(Z_l) for its own
//                backward pass.
//   k_train_dw   one thread-block cluster per tile of a weight matrix: the CTAs of
//                the cluster split the minibatch's row tiles, each accumulates
//                dW = dZ^T X over its rows in tensor memory, the partials are
//                summed over the cluster through distributed shared memory in a
//                fixed order (so a step is deterministic), and each CTA applies
//                AdamW to its share of the tile and refreshes the BF16 images.
//
// The bias rides in the GEMMs: every layer input carries a column of ones after
// its features (X_aug = [X | 1 | 0 ...], K padded to 16), and the weights are kept
// augmented, W_aug = [W | b | 0 ...] (rows padded to 16), so the forward product
// already holds the bias and the weight gradient's ones column is the bias
// gradient.
//
// A tcgen05.mma of M = 128 occupies the tensor pipe for about as long at N = 64 as
// at N = 256 (measured: ~130 cycles either way), so every GEMM here runs the full
// layer width per instruction.  Operand layout: K-major core matrices (8 rows x
// 16 bytes; core (row/8, k/8) of a block of width w at ((row/8) * (w/8) + k/8) *
// 128 bytes):
//   * an activation image X (128 rows x K_aug) and a gradient image dZ (128 rows
//     x N_pad) are one block each;
//   * the forward weights W_aug (N_pad x K_aug) are slabs of 32 input columns
//     with all output rows (one bulk copy, the B operand of N_pad-wide MMAs);
//   * the input-gradient GEMM reads W^T (d_in x N_pad), kept as slabs of 32
//     outputs with all d_in rows, so it too runs d_in-wide MMAs.
// The weight-gradient GEMM reads the X and dZ images of the row tiles through
// MN-major descriptors (k = rows; the stride byte offset is the core stride along
// M/N, the leading byte offset the stride between groups of 8 along K), so no
// transposed activation is ever written.
//
// Every mbarrier wait is bounded (on a timeout the thread records an error and
// skips the work that depended on it, but still arrives everywhere it is
// expected); there is no counterpart in the reference (its pipeline has no
// learned part).
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <math_constants.h>
#include <stdint.h>

#include <cmath>

#include "pb_gelu.cuh"
#include "pybasin_b200.h"

namespace {

constexpr int kRows = 128;                 // rows of a tile = MMA M = TMEM lanes
constexpr int kMaxLayers = PB_TRAIN_MAX_LAYERS;
constexpr int kMaxWidth = 256;             // largest layer width
constexpr int kMaxPieces = 4;              // 64-column pieces of a layer output (<= 256)
constexpr int kMaxKaug = 272;
constexpr int kMaxClasses = 32;            // the cross entropy reads one 32-column TMEM load
constexpr long long kWaitPolls = 1ll << 22;

// k_train_fb: 16 epilogue warps (TMEM lane quarter w % 4, output piece w / 4),
// one MMA-issuing warp, one warp streaming the weight slabs
constexpr int kEpiWarps = 16;
constexpr int kMmaWarp = kEpiWarps;
constexpr int kLoadWarp = kEpiWarps + 1;               // the first copy-issuing warp
// Bulk copies issued by one thread follow each other (about a microsecond each,
// whatever the size up to ~100 KB); copies from different warps overlap, so the
// weight copies are dealt round robin to kLoadWarps warps
#ifndef PB_LOAD_WARPS
#define PB_LOAD_WARPS 1
#endif
constexpr int kLoadWarps = PB_LOAD_WARPS;
constexpr int kFbThreads = (kEpiWarps + 1 + kLoadWarps) * 32;
constexpr int kSlabBytes = 16 * 1024;                    // a weight slab: all rows x as many columns as fit
// A bulk copy costs about the same whatever its size up to tens of KB, so the
// slabs stream in groups of consecutive slabs (contiguous in the image), one copy
// per group, into ring slots of kGroup slabs
#ifndef PB_FB_GROUP
#define PB_FB_GROUP 3
#endif
#ifndef PB_FB_RING
#define PB_FB_RING 3
#endif
constexpr int kGroup = PB_FB_GROUP;                      // slabs per copy
constexpr int kRing = PB_FB_RING;                        // slots of the weight ring
constexpr int kSlotBytes = kGroup * kSlabBytes;
constexpr int kImgBytes = kRows * kMaxKaug * 2;          // largest activation / gradient image
constexpr int kFbTail = 1024;                            // barriers, flags, the tile's labels
constexpr int kFbSmem = kImgBytes + kRing * kSlotBytes + kFbTail;

// k_train_dw
#ifndef PB_DW_PRODUCERS
#define PB_DW_PRODUCERS 4
#endif
constexpr int kDwProducers = PB_DW_PRODUCERS;
// the MMA warp and the producers, in whole groups of four warps (the TMEM readout
// gives each warp a lane quarter), at least eight warps
constexpr int kDwThreads = ((kDwProducers + 1 + 3) / 4 * 4 > 8 ? (kDwProducers + 1 + 3) / 4 * 4 : 8) * 32;
constexpr int kDwStages = 3;
constexpr int kDwMaxIn = 144;                       // inputs of a weight tile
constexpr int kDwABytes = kRows * kRows * 2;        // 128 outputs x 128 rows
constexpr int kDwBBytes = kRows * kDwMaxIn * 2;     // 128 rows x <= 144 inputs
constexpr int kDwStageBytes = kDwABytes + kDwBBytes;
constexpr int kDwTail = 256;
constexpr int kDwSmem = kDwStages * kDwStageBytes + kDwTail;
constexpr int kMaxCluster = 8;
// warps 1 .. kDwProducers copy the row groups of a stage, 16 / kDwProducers each:
// the lanes of one warp issue their copies together, but at about 26 B/clk for
// 2 KB copies; copies from several warps proceed side by side
static_assert(16 % kDwProducers == 0 && kDwProducers + 1 <= kDwThreads / 32, "k_train_dw: producer warps");
constexpr int kMaxDwTiles = kMaxLayers * 2 * 2;  // per layer <= 2 output tiles x 2 input ranges

// ---- geometry ----------------------------------------------------------------

struct LayerGeo {
    int din, dout;        // real widths
    int kaug;             // K of the forward GEMM: din + 1 (ones) rounded up to 16
    int npad;             // output rows padded to 16
    int n_pieces;         // 64-column pieces of npad (forward outputs)
    int p0[kMaxPieces], ph[kMaxPieces];
    int n_dx;             // 64-column pieces of din (input-gradient outputs, layers >= 1)
    int d0[kMaxPieces], dw[kMaxPieces];
    int sw;               // input columns of a W slab (all npad rows; <= kSlabBytes)
    int tw;               // outputs of a W^T slab (all din rows; <= kSlabBytes)
    int64_t w_off;        // byte offset of this layer's W slabs in the image buffer
    int64_t wt_off;       // byte offset of its W^T slabs (layers >= 1)
    int64_t aug_off;      // element offset of this layer in the concatenated augmented (npad x kaug) arrays
    int64_t x_off, z_off, g_off;     // byte offsets in the scratch of the layer's X / dZ / GELU' images (tile 0)
    int64_t x_tile, z_tile, g_tile;  // bytes per row tile
};

struct Geo {
    int n_layers, tiles;
    LayerGeo l[kMaxLayers];
    int64_t img_bytes, scratch_bytes, aug_elems;
};

__host__ __device__ inline int split64(int n, int* o0, int* w)
{
    int k = 0;
    for (int o = 0; o < n; o += 64) {
        o0[k] = o;
        w[k] = n - o < 64 ? n - o : 64;
        ++k;
    }
    return k;
}

inline int geo_build(int n_layers, const int32_t* dims, int batch, Geo* g)
{
    if (n_layers < 1 || n_layers > kMaxLayers || batch < 1 || !dims) return PB_EINVAL;
    if (dims[0] < 8 || dims[0] > kMaxWidth || dims[0] % 8) return PB_EINVAL;
    for (int l = 1; l < n_layers; ++l)
        if (dims[l] < 16 || dims[l] > kMaxWidth || dims[l] % 16) return PB_EINVAL;
    if (dims[n_layers] < 2 || dims[n_layers] > kMaxClasses) return PB_EINVAL;
    g->n_layers = n_layers;
    g->tiles = (batch + kRows - 1) / kRows;
    int64_t img = 0, aug = 0, scr = 0;
    for (int l = 0; l < n_layers; ++l) {
        LayerGeo& L = g->l[l];
        L.din = dims[l];
        L.dout = dims[l + 1];
        L.kaug = (L.din + 1 + 15) / 16 * 16;
        L.npad = (L.dout + 15) / 16 * 16;
        L.n_pieces = split64(L.npad, L.p0, L.ph);
        L.n_dx = l > 0 ? split64(L.din, L.d0, L.dw) : 0;
        // slab widths: as many 16-column groups as fit kSlabBytes (at least one)
        L.sw = min(L.kaug, max(16, kSlabBytes / (2 * L.npad) / 16 * 16));
        L.tw = min(L.npad, max(16, kSlabBytes / (2 * L.din) / 16 * 16));
        L.w_off = img;
        img += static_cast<int64_t>(L.npad) * L.kaug * 2;
        L.wt_off = img;
        if (l > 0) img += static_cast<int64_t>(L.din) * L.npad * 2;
        L.aug_off = aug;
        aug += static_cast<int64_t>(L.npad) * L.kaug;
        L.x_tile = static_cast<int64_t>(kRows) * L.kaug * 2;
        L.z_tile = static_cast<int64_t>(kRows) * L.npad * 2;
        L.g_tile = l + 1 < n_layers ? static_cast<int64_t>(kRows) * L.dout * 2 : 0;
    }
    for (int l = 0; l < n_layers; ++l) {
        LayerGeo& L = g->l[l];
        L.x_off = scr;
        scr += L.x_tile * g->tiles;
        L.z_off = scr;
        scr += L.z_tile * g->tiles;
        L.g_off = scr;
        scr += L.g_tile * g->tiles;
    }
    g->img_bytes = img;
    g->aug_elems = aug;
    g->scratch_bytes = scr;
    return PB_SUCCESS;
}

// byte offset of element (r, k) in a single-block image of width w
__host__ __device__ __forceinline__ uint32_t img_off(int w, int r, int k)
{
    return static_cast<uint32_t>((((r >> 3) * (w >> 3) + (k >> 3)) << 7) + ((r & 7) << 4) + ((k & 7) << 1));
}

// byte offset (relative to the layer's W slabs) of weight element (o, i): slab
// i / sw holds all npad rows of sw (the last one fewer) columns
__host__ __device__ inline int64_t w_elem(const LayerGeo& L, int o, int i)
{
    const int k0 = i / L.sw * L.sw, kw = min(L.sw, L.kaug - k0);
    return static_cast<int64_t>(L.npad) * k0 * 2 + img_off(kw, o, i - k0);
}

// byte offset (relative to the layer's W^T slabs) of weight element (o, i), i < din:
// slab o / tw holds all din rows of W^T for tw (the last one fewer) outputs
__host__ __device__ inline int64_t wt_elem(const LayerGeo& L, int o, int i)
{
    const int o0 = o / L.tw * L.tw, ow = min(L.tw, L.npad - o0);
    return static_cast<int64_t>(L.din) * o0 * 2 + img_off(ow, i, o - o0);
}

// ---- device helpers ----------------------------------------------------------

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// shared-memory matrix descriptor: start, leading / stride byte offsets (16-byte
// units), version 1, base offset 0, no swizzle
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    return static_cast<uint64_t>((addr >> 4) & 0x3FFFu) | (static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16) |
           (static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// kind::f16 instruction descriptor: FP32 accumulator, BF16 A and B; a_mn / b_mn
// select the MN-major (transposed) operand layouts
__device__ __forceinline__ uint32_t instr_desc(int M, int N, bool a_mn, bool b_mn)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | (a_mn ? 1u << 15 : 0u) | (b_mn ? 1u << 16 : 0u) |
           (static_cast<uint32_t>(N >> 3) << 17) | (static_cast<uint32_t>(M >> 4) << 24);
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

// waits for the phase of the given parity; gives up (false) after kWaitPolls polls
// or at once when *abort is set
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int* abort)
{
    for (long long i = 0; i < kWaitPolls; ++i) {
        if (mbar_try(bar, parity)) return true;
        if ((i & 1023) == 1023 && *abort) return false;
    }
    *abort = 1;
    return false;
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void bulk_load(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

__device__ __forceinline__ void bulk_store(void* dst, uint32_t src, uint32_t bytes)
{
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(src), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void bulk_wait_read()
{
    asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N) : "memory");
}
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

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

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// 64 columns: two loads in flight, one wait
__device__ __forceinline__ void tmem_ld64(uint32_t taddr, uint32_t (&v)[64])
{
#pragma unroll
    for (int h = 0; h < 2; ++h)
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
            "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
            "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
            : "=r"(v[32 * h + 0]), "=r"(v[32 * h + 1]), "=r"(v[32 * h + 2]), "=r"(v[32 * h + 3]), "=r"(v[32 * h + 4]),
              "=r"(v[32 * h + 5]), "=r"(v[32 * h + 6]), "=r"(v[32 * h + 7]), "=r"(v[32 * h + 8]), "=r"(v[32 * h + 9]),
              "=r"(v[32 * h + 10]), "=r"(v[32 * h + 11]), "=r"(v[32 * h + 12]), "=r"(v[32 * h + 13]),
              "=r"(v[32 * h + 14]), "=r"(v[32 * h + 15]), "=r"(v[32 * h + 16]), "=r"(v[32 * h + 17]),
              "=r"(v[32 * h + 18]), "=r"(v[32 * h + 19]), "=r"(v[32 * h + 20]), "=r"(v[32 * h + 21]),
              "=r"(v[32 * h + 22]), "=r"(v[32 * h + 23]), "=r"(v[32 * h + 24]), "=r"(v[32 * h + 25]),
              "=r"(v[32 * h + 26]), "=r"(v[32 * h + 27]), "=r"(v[32 * h + 28]), "=r"(v[32 * h + 29]),
              "=r"(v[32 * h + 30]), "=r"(v[32 * h + 31])
            : "r"(taddr + 32u * h));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// All threads of the CTA, in the non-aligned form (warps may arrive diverged:
// one lane issued the MMAs or the copies)
__device__ __forceinline__ void cta_sync() { asm volatile("barrier.sync 0;" ::: "memory"); }

__device__ __forceinline__ void mbar_arrive(uint32_t bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tc_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void proxy_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ uint32_t pack_bf16(float a, float b)
{
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t*>(&h);
}

__device__ __forceinline__ uint32_t pack_f16(float a, float b)
{
    const __half2 h = __floats2half2_rn(a, b);
    return *reinterpret_cast<const uint32_t*>(&h);
}

__device__ __forceinline__ float2 unpack_f16(uint32_t u)
{
    return __half22float2(*reinterpret_cast<const __half2*>(&u));
}

using pb::gelu;
using pb::gelu_grad;

}  // namespace

namespace {

// GELU and its derivative sharing one tanh (the forms of pb_gelu.cuh)
__device__ __forceinline__ void gelu_both(float x, float& g, float& d)
{
    const float x2 = x * x;
    const float t = pb::tanh_approx(x * fmaf(pb::kGeluB, x2, pb::kGeluA));
    const float hx = 0.5f * x;
    g = fmaf(hx, t, hx);
    const float du = fmaf(pb::kGeluB3, x2, pb::kGeluA);
    d = fmaf(hx * du, fmaf(-t, t, 1.f), 0.5f * (1.f + t));
}

struct FbArgs {
    Geo geo;
    const __nv_bfloat16* x;  // training inputs (n_rows x dims[0]) BF16
    const int32_t* labels;   // (n_rows)
    const int32_t* rows;     // the minibatch's rows of x (M)
    int n_rows;              // rows of x (and labels)
    int M;
    float scale;             // 1 / M: the loss is the minibatch mean
    const uint8_t* w_img;    // BF16 weight slabs, all layers
    uint8_t* scratch;        // X / dZ / GELU' images of the minibatch's row tiles
    float* loss_sum;
    int32_t* correct;
    int32_t* error;
};

// full / empty: the weight-slab ring; mdone: the MMAs of a phase are done;
// epi_done: every epilogue warp finished the phase (the MMA warp starts the next)
struct FbSmem {
    uint64_t full[kRing], empty[kRing], mdone, epi_done;
    uint32_t tmem;
    int abort;
    int y[kRows];
};
static_assert(sizeof(FbSmem) <= kFbTail, "k_train_fb: barrier block");
static_assert(kFbSmem <= 227 * 1024, "k_train_fb: shared memory");

// Epilogue of one forward piece of a hidden layer: z (TMEM columns col0 .. col0 +
// ncols) -> GELU(z) into the next layer's input image (width wn), GELU'(z) (FP16)
// to global.
__device__ __forceinline__ void fwd_hidden_cols(uint32_t tm, int ncols, int col0, int r, uint8_t* xo, int wn,
                                                uint8_t* gimg)
{
    for (int cc = 0; cc < ncols; cc += 32) {
        const int n = ncols - cc >= 32 ? 32 : 16;
        float z[32];
        if (n == 32) {
            uint32_t v[32];
            tmem_ld32(tm + static_cast<uint32_t>(cc), v);
#pragma unroll
            for (int j = 0; j < 32; ++j) z[j] = __uint_as_float(v[j]);
        } else {
            uint32_t v[16];
            tmem_ld16(tm + static_cast<uint32_t>(cc), v);
#pragma unroll
            for (int j = 0; j < 16; ++j) z[j] = __uint_as_float(v[j]);
#pragma unroll
            for (int j = 16; j < 32; ++j) z[j] = 0.f;
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            if (q * 8 >= n) break;
            uint32_t hx[4], hd[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                float g0, d0, g1, d1;
                gelu_both(z[q * 8 + 2 * k], g0, d0);
                gelu_both(z[q * 8 + 2 * k + 1], g1, d1);
                hx[k] = pack_bf16(g0, g1);
                hd[k] = pack_f16(d0, d1);
            }
            const int col = col0 + cc + q * 8;
            *reinterpret_cast<uint4*>(xo + img_off(wn, r, col)) = make_uint4(hx[0], hx[1], hx[2], hx[3]);
            *reinterpret_cast<uint4*>(gimg + ((static_cast<int64_t>(col >> 3) * kRows + r) << 4)) =
                make_uint4(hd[0], hd[1], hd[2], hd[3]);
        }
    }
}

// Epilogue of one input-gradient piece: dZ_below = acc * GELU'(Z_below) (TMEM
// columns col0 .. col0 + ncols) into the gradient image (width wb) of the layer below.
__device__ __forceinline__ void dx_cols(uint32_t tm, int ncols, int col0, int r, uint8_t* zo, int wb,
                                        const uint8_t* gimg)
{
    for (int cc = 0; cc < ncols; cc += 32) {
        const int n = ncols - cc >= 32 ? 32 : 16;
        uint4 gd[4];
#pragma unroll
        for (int q = 0; q < 4; ++q)
            if (q * 8 < n)
                gd[q] = __ldg(reinterpret_cast<const uint4*>(
                    gimg + ((static_cast<int64_t>((col0 + cc) / 8 + q) * kRows + r) << 4)));
        float a[32];
        if (n == 32) {
            uint32_t v[32];
            tmem_ld32(tm + static_cast<uint32_t>(cc), v);
#pragma unroll
            for (int j = 0; j < 32; ++j) a[j] = __uint_as_float(v[j]);
        } else {
            uint32_t v[16];
            tmem_ld16(tm + static_cast<uint32_t>(cc), v);
#pragma unroll
            for (int j = 0; j < 16; ++j) a[j] = __uint_as_float(v[j]);
#pragma unroll
            for (int j = 16; j < 32; ++j) a[j] = 0.f;
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            if (q * 8 >= n) break;
            const uint32_t gw[4] = {gd[q].x, gd[q].y, gd[q].z, gd[q].w};
            uint32_t h[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const float2 d = unpack_f16(gw[k]);
                h[k] = pack_bf16(a[q * 8 + 2 * k] * d.x, a[q * 8 + 2 * k + 1] * d.y);
            }
            *reinterpret_cast<uint4*>(zo + img_off(wb, r, col0 + cc + q * 8)) = make_uint4(h[0], h[1], h[2], h[3]);
        }
    }
}

__global__ void __launch_bounds__(kFbThreads, 1) k_train_fb(const __grid_constant__ FbArgs p)
{
    extern __shared__ __align__(1024) uint8_t smem[];
    // the image buffer (each phase's epilogue overwrites its input in place), then
    // the slab ring, then FbSmem
    uint8_t* ring = smem + kImgBytes;
    FbSmem* sh = reinterpret_cast<FbSmem*>(ring + kRing * kSlotBytes);
    volatile int* abort = &sh->abort;
    const Geo& G = p.geo;
    const int NL = G.n_layers;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int tile = blockIdx.x;
    const int m0 = tile * kRows;
    const int mt = min(kRows, p.M - m0);  // valid rows of this tile

    if (tid == 0) {
        for (int s = 0; s < kRing; ++s) {
            mbar_init(smem_u32(&sh->full[s]), 1);
            mbar_init(smem_u32(&sh->empty[s]), 1);
        }
        mbar_init(smem_u32(&sh->mdone), 1);
        mbar_init(smem_u32(&sh->epi_done), kEpiWarps);
        sh->abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&sh->tmem)),
                     "r"(256)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_before();
    cta_sync();
    tc_after();
    const uint32_t tmem = sh->tmem;

    if (warp >= kLoadWarp) {
        // ---- weight slabs into the ring, in the order the MMA warp consumes them:
        // forward W slabs of every layer, then the W^T slabs from the last layer down;
        // copy u is issued by load warp u % kLoadWarps
        if (lane == 0) {
            const uint32_t lw = static_cast<uint32_t>(warp - kLoadWarp);
            uint32_t u = 0;
            auto put = [&](int64_t off, uint32_t bytes) {
                const uint32_t s = u % kRing, round = u / kRing;
                if (u++ % kLoadWarps != lw) return;
                if (round > 0 && !mbar_wait(smem_u32(&sh->empty[s]), (round - 1) & 1u, abort)) return;
                mbar_expect_tx(smem_u32(&sh->full[s]), bytes);
                bulk_load(smem_u32(ring + s * kSlotBytes), p.w_img + off, bytes, smem_u32(&sh->full[s]));
            };
            for (int l = 0; l < NL && !*abort; ++l) {
                const LayerGeo& L = G.l[l];
                for (int g0 = 0; g0 < L.kaug; g0 += kGroup * L.sw)
                    put(L.w_off + static_cast<int64_t>(L.npad) * g0 * 2,
                        static_cast<uint32_t>(L.npad) * min(kGroup * L.sw, L.kaug - g0) * 2u);
            }
            for (int l = NL - 1; l >= 1 && !*abort; --l) {
                const LayerGeo& L = G.l[l];
                for (int g0 = 0; g0 < L.npad; g0 += kGroup * L.tw)
                    put(L.wt_off + static_cast<int64_t>(L.din) * g0 * 2,
                        static_cast<uint32_t>(L.din) * min(kGroup * L.tw, L.npad - g0) * 2u);
            }
        }
        __syncwarp();
        cta_sync();
        if (tid == kLoadWarp * 32 && *abort && p.error) atomicExch(p.error, 1);
        return;
    }

    if (warp == kMmaWarp) {
        // ---- MMAs, one phase per layer: the previous phase's epilogues are done and
        // the image they wrote is final; its copy to global scratch (for the weight
        // gradients) starts, the MMAs read it, and before the phase's epilogues may
        // overwrite it the copy has read it (it overlaps the MMAs)
        if (lane == 0) {
            uint32_t u = 0, ep = 0;
            const uint32_t a0 = smem_u32(smem);
            auto begin_phase = [&](uint8_t* dst, uint32_t bytes) {
                mbar_wait(smem_u32(&sh->epi_done), ep++ & 1u, abort);
                tc_after();
                bulk_store(dst, a0, bytes);
                bulk_commit();
            };
            auto end_mmas = [&]() {
                bulk_wait_read<0>();
                mma_commit(smem_u32(&sh->mdone));
            };
            auto slab = [&](uint32_t& s) {
                s = u % kRing;
                const uint32_t round = u / kRing;
                ++u;
                const bool ok = mbar_wait(smem_u32(&sh->full[s]), round & 1u, abort);
                tc_after();
                return ok;
            };
            for (int l = 0; l < NL; ++l) {  // forward: Z_l (128 x npad) = X_l W_l^T, K = kaug
                const LayerGeo& L = G.l[l];
                begin_phase(p.scratch + L.x_off + tile * L.x_tile, static_cast<uint32_t>(L.x_tile));
                const uint32_t sbo_a = static_cast<uint32_t>(L.kaug >> 3) << 7;
                const uint32_t idesc = instr_desc(kRows, L.npad, false, false);
                for (int g0 = 0; g0 < L.kaug; g0 += kGroup * L.sw) {
                    uint32_t s;
                    const bool ok = slab(s);
                    const uint32_t sb = smem_u32(ring + s * kSlotBytes);
                    for (int k0 = g0; ok && k0 < min(g0 + kGroup * L.sw, L.kaug); k0 += L.sw) {
                        const int kw = min(L.sw, L.kaug - k0);
                        const uint32_t b0 = sb + static_cast<uint32_t>(L.npad * (k0 - g0) * 2);
                        const uint32_t sbo_b = static_cast<uint32_t>(kw >> 3) << 7;
                        for (int ks = 0; ks < (kw >> 4); ++ks)
                            mma_bf16(tmem, smem_desc(a0 + ((k0 >> 3) + 2 * ks) * 128u, 128u, sbo_a),
                                     smem_desc(b0 + ks * 256u, 128u, sbo_b), idesc, (k0 > 0 || ks > 0) ? 1u : 0u);
                    }
                    mma_commit(smem_u32(&sh->empty[s]));
                }
                end_mmas();
            }
            for (int l = NL - 1; l >= 1; --l) {  // input gradients: (128 x din) = dZ_l W_l, K = npad
                const LayerGeo& L = G.l[l];
                begin_phase(p.scratch + L.z_off + tile * L.z_tile, static_cast<uint32_t>(L.z_tile));
                const uint32_t sbo_a = static_cast<uint32_t>(L.npad >> 3) << 7;
                const uint32_t idesc = instr_desc(kRows, L.din, false, false);
                for (int g0 = 0; g0 < L.npad; g0 += kGroup * L.tw) {
                    uint32_t s;
                    const bool ok = slab(s);
                    const uint32_t sb = smem_u32(ring + s * kSlotBytes);
                    for (int o0 = g0; ok && o0 < min(g0 + kGroup * L.tw, L.npad); o0 += L.tw) {
                        const int ow = min(L.tw, L.npad - o0);
                        const uint32_t b0 = sb + static_cast<uint32_t>(L.din * (o0 - g0) * 2);
                        const uint32_t sbo_b = static_cast<uint32_t>(ow >> 3) << 7;
                        for (int ks = 0; ks < (ow >> 4); ++ks)
                            mma_bf16(tmem, smem_desc(a0 + ((o0 >> 3) + 2 * ks) * 128u, 128u, sbo_a),
                                     smem_desc(b0 + ks * 256u, 128u, sbo_b), idesc, (o0 > 0 || ks > 0) ? 1u : 0u);
                    }
                    mma_commit(smem_u32(&sh->empty[s]));
                }
                end_mmas();
            }
            // the last image written (dZ_0) to scratch once its phase is done
            mbar_wait(smem_u32(&sh->epi_done), ep++ & 1u, abort);
            bulk_store(p.scratch + G.l[0].z_off + tile * G.l[0].z_tile, a0, static_cast<uint32_t>(G.l[0].z_tile));
            bulk_commit();
            bulk_wait_all();
        }
        __syncwarp();
    } else {
        // ---- epilogue warps: the inputs of the row tile first (rows of x by the
        // minibatch's indices, the ones column after them, zero rows past the minibatch)
        const LayerGeo& L0 = G.l[0];
        const int pieces = L0.kaug >> 3;
        for (int idx = tid; idx < kRows * pieces; idx += kEpiWarps * 32) {
            const int r = idx & (kRows - 1), col = (idx >> 7) << 3;
            uint8_t* dst = smem + img_off(L0.kaug, r, col);
            const int row = r < mt ? __ldg(p.rows + m0 + r) : -1;
            const bool in_range = row >= 0 && row < p.n_rows;
            if (r < mt && !in_range && col == 0) sh->abort = 1;  // a row index outside x: reported, not read
            if (in_range && col < L0.din) {
                const int64_t src = static_cast<int64_t>(row) * L0.din + col;
                asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(p.x + src) : "memory");
            } else {
                const uint32_t one = (r < mt && col == L0.din) ? 0x3F80u : 0u;  // BF16 1.0 in the first slot
                *reinterpret_cast<uint4*>(dst) = make_uint4(one, 0u, 0u, 0u);
            }
        }
        for (int r = tid; r < kRows; r += kEpiWarps * 32) {
            const int row = r < mt ? __ldg(p.rows + m0 + r) : -1;
            sh->y[r] = (row >= 0 && row < p.n_rows) ? __ldg(p.labels + row) : -1;
        }
        asm volatile("cp.async.wait_all;" ::: "memory");
        proxy_fence();
        __syncwarp();
        if (lane == 0) mbar_arrive(smem_u32(&sh->epi_done));

        const int quarter = warp & 3, grp = warp >> 2;
        const int r = quarter * 32 + lane;  // this thread's row (TMEM lane)
        const uint32_t tm_row = tmem + (static_cast<uint32_t>(quarter * 32) << 16);
        uint32_t ph = 1;                    // this phase (the gather was phase 0)
        float loss = 0.f;
        int hits = 0;
        // one phase of the epilogue.  Every warp waits for the phase's MMAs (mdone
        // completes once per phase, and a wait by parity cannot tell phases two
        // apart, so no warp may skip one), works on its piece if it has one, and
        // arrives on epi_done.
        auto end_phase = [&](bool worked) {
            if (worked) {
                proxy_fence();
                tc_before();
            } else if (lane == 0) {
                mbar_wait(smem_u32(&sh->mdone), (ph - 1) & 1u, abort);
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_u32(&sh->epi_done));
            ++ph;
        };
        for (int l = 0; l < NL; ++l) {
            const LayerGeo& L = G.l[l];
            const bool last = l + 1 == NL;
            const bool mine = last ? grp == 0 : grp < L.n_pieces;
            if (mine) {
                const bool ok = __all_sync(0xffffffffu, mbar_wait(smem_u32(&sh->mdone), (ph - 1) & 1u, abort));
                tc_after();
                uint8_t* out = smem;  // in place: the phase's MMAs are done with their input
                if (!last) {
                    const LayerGeo& Ln = G.l[l + 1];
                    const int pc = grp;
                    if (ok)
                        fwd_hidden_cols(tm_row + static_cast<uint32_t>(L.p0[pc]), L.ph[pc], L.p0[pc], r, out, Ln.kaug,
                                        p.scratch + L.g_off + tile * L.g_tile);
                    if (pc == L.n_pieces - 1) {
                        // the ones column of the next layer's input, then zeros to its K
                        for (int col = L.dout; col < Ln.kaug; col += 8) {
                            const uint32_t one = (r < mt && col == L.dout) ? 0x3F80u : 0u;
                            *reinterpret_cast<uint4*>(out + img_off(Ln.kaug, r, col)) = make_uint4(one, 0u, 0u, 0u);
                        }
                    }
                } else {
                    // softmax cross entropy of the logits (TMEM columns 0 .. npad)
                    uint32_t v[32];
                    if (ok) tmem_ld32(tm_row, v);
                    const int C = L.dout;
                    const int y = sh->y[r];
                    float z[32];
                    float mx = -CUDART_INF_F, zy = 0.f;
                    int arg = 0;
#pragma unroll
                    for (int c = 0; c < 32; ++c) {
                        z[c] = __uint_as_float(v[c]);
                        if (c < C && z[c] > mx) {
                            mx = z[c];
                            arg = c;
                        }
                        if (c == y) zy = z[c];
                    }
                    float se = 0.f;
#pragma unroll
                    for (int c = 0; c < 32; ++c) {
                        z[c] = c < C ? __expf(z[c] - mx) : 0.f;
                        se += z[c];
                    }
                    const float inv = 1.f / se;
                    const bool valid = r < mt && ok;
#pragma unroll
                    for (int c8 = 0; c8 < 32; c8 += 8) {
                        if (c8 >= L.npad) break;
                        uint32_t h[4];
#pragma unroll
                        for (int k = 0; k < 4; ++k) {
                            const int c = c8 + 2 * k;
                            const float d0 = valid ? (z[c] * inv - (c == y ? 1.f : 0.f)) * p.scale : 0.f;
                            const float d1 = valid ? (z[c + 1] * inv - (c + 1 == y ? 1.f : 0.f)) * p.scale : 0.f;
                            h[k] = pack_bf16(d0, d1);
                        }
                        *reinterpret_cast<uint4*>(out + img_off(L.npad, r, c8)) = make_uint4(h[0], h[1], h[2], h[3]);
                    }
                    if (valid && y >= 0 && y < C) {
                        loss = -(zy - mx - __logf(se));
                        hits = arg == y ? 1 : 0;
                    }
                }
            }
            end_phase(mine);
        }
        for (int l = NL - 1; l >= 1; --l) {
            const LayerGeo& L = G.l[l];
            const LayerGeo& Lb = G.l[l - 1];
            const bool mine = grp < L.n_dx;
            if (mine) {
                const bool ok = __all_sync(0xffffffffu, mbar_wait(smem_u32(&sh->mdone), (ph - 1) & 1u, abort));
                tc_after();
                if (ok)
                    dx_cols(tm_row + static_cast<uint32_t>(L.d0[grp]), L.dw[grp], L.d0[grp], r,
                            smem, Lb.npad, p.scratch + Lb.g_off + tile * Lb.g_tile);
            }
            end_phase(mine);
        }
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) {
            loss += __shfl_xor_sync(0xffffffffu, loss, o);
            hits += __shfl_xor_sync(0xffffffffu, hits, o);
        }
        if (lane == 0 && grp == 0) {
            if (p.loss_sum && loss != 0.f) atomicAdd(p.loss_sum, loss);
            if (p.correct && hits) atomicAdd(p.correct, hits);
        }
    }
    tc_before();
    cta_sync();
    __syncwarp();
    if (tid == 0 && *abort && p.error) atomicExch(p.error, 1);
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(256) : "memory");
}

// ---- inference: two row tiles per CTA in turn ----------------------------------
//
// A persistent CTA takes pairs of 128-row tiles and runs the layer chain of both,
// alternating: the MMAs of one tile's layer run while the epilogue warps apply
// GELU to the other tile's previous layer, so the tensor pipe and the epilogue
// overlap.  Activations stay in shared memory (one buffer per tile, overwritten in
// place), the accumulators in TMEM (256 columns per tile), the weights (the same
// augmented slab images as the training step) stream through the slab ring once
// per tile and layer.  The logits of the last layer go to global memory.
struct InferArgs {
    Geo geo;
    const __nv_bfloat16* x;  // (n x dims[0]) BF16 inputs
    int64_t n;
    const uint8_t* w_img;
    float* logits;           // (n x C)
    int32_t* error;
};

#ifndef PB_INF_GROUP
#define PB_INF_GROUP 2
#endif
#ifndef PB_INF_RING
#define PB_INF_RING 2
#endif
constexpr int kInfGroup = PB_INF_GROUP;  // slabs per copy
constexpr int kInfRing = PB_INF_RING;
constexpr int kInfSlot = kInfGroup * kSlabBytes;
constexpr int kInfSmem = 2 * kImgBytes + kInfRing * kInfSlot + 1024;
static_assert(kInfSmem <= 227 * 1024, "k_mlp_infer_pp: shared memory");

struct InfSmem {
    uint64_t full[kInfRing], empty[kInfRing], mdone[2], edone[2];
    uint32_t tmem;
    int abort;
};

// rows [row0, row0 + 128) of x into the layer-0 image at img: the ones column
// after the inputs, zeros past n (run by the 16 epilogue warps)
__device__ __forceinline__ void infer_stage(const InferArgs& p, const LayerGeo& L0, uint8_t* img, int64_t row0, int tid)
{
    const int pieces = L0.kaug >> 3;
    for (int idx = tid; idx < kRows * pieces; idx += kEpiWarps * 32) {
        const int r = idx & (kRows - 1), col = (idx >> 7) << 3;
        uint8_t* dst = img + img_off(L0.kaug, r, col);
        const int64_t row = row0 + r;
        if (row < p.n && col < L0.din) {
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(p.x + row * L0.din + col)
                         : "memory");
        } else {
            const uint32_t one = (row < p.n && col == L0.din) ? 0x3F80u : 0u;
            *reinterpret_cast<uint4*>(dst) = make_uint4(one, 0u, 0u, 0u);
        }
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
}

// GELU of NN accumulator columns of row r into the next layer's image (width w)
// at columns col .. col + NN
template <int NN>
__device__ __forceinline__ void gelu_cols(const uint32_t (&v)[NN], uint8_t* act, int w, int r, int col)
{
#pragma unroll
    for (int q = 0; q < NN / 8; ++q) {
        uint32_t hx[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            float g0, g1;
            pb::gelu2(__uint_as_float(v[q * 8 + 2 * k]), __uint_as_float(v[q * 8 + 2 * k + 1]), g0, g1);
            hx[k] = pack_bf16(g0, g1);
        }
        *reinterpret_cast<uint4*>(act + img_off(w, r, col + q * 8)) = make_uint4(hx[0], hx[1], hx[2], hx[3]);
    }
}

__global__ void __launch_bounds__(kFbThreads, 1) k_mlp_infer_pp(const __grid_constant__ InferArgs p)
{
    extern __shared__ __align__(1024) uint8_t smem[];
    // the activations of tile t at smem + t * kImgBytes, then the slab ring
    uint8_t* ring = smem + 2 * kImgBytes;
    InfSmem* sh = reinterpret_cast<InfSmem*>(ring + kInfRing * kInfSlot);
    volatile int* abort = &sh->abort;
    const Geo& G = p.geo;
    const int NL = G.n_layers;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int64_t n_tiles = (p.n + kRows - 1) / kRows, n_pairs = (n_tiles + 1) / 2;

    if (tid == 0) {
        for (int s = 0; s < kInfRing; ++s) {
            mbar_init(smem_u32(&sh->full[s]), 1);
            mbar_init(smem_u32(&sh->empty[s]), 1);
        }
        for (int t = 0; t < 2; ++t) {
            mbar_init(smem_u32(&sh->mdone[t]), 1);
            mbar_init(smem_u32(&sh->edone[t]), kEpiWarps);
        }
        sh->abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&sh->tmem)),
                     "r"(512)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_before();
    cta_sync();
    tc_after();
    const uint32_t tmem = sh->tmem;

    if (warp >= kLoadWarp) {
        if (lane == 0) {  // the slabs of every layer, once per tile, in the MMA order; copy u by load warp u % kLoadWarps
            const uint32_t lw = static_cast<uint32_t>(warp - kLoadWarp);
            uint32_t u = 0;
            for (int64_t pr = blockIdx.x; pr < n_pairs && !*abort; pr += gridDim.x) {
                // the next pair's input rows into L2: the epilogue stages them at the
                // end of this pair
                const int64_t nxt = pr + gridDim.x;
                if (lw == 0 && nxt < n_pairs) {
                    const int64_t r0 = 2 * nxt * kRows, r1 = min(p.n, r0 + 2 * kRows);
                    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p.x + r0 * G.l[0].din),
                                 "r"(static_cast<uint32_t>((r1 - r0) * G.l[0].din * 2)) : "memory");
                }
                for (int l = 0; l < NL; ++l)
                    for (int t = 0; t < 2; ++t) {
                        const LayerGeo& L = G.l[l];
                        for (int g0 = 0; g0 < L.kaug; g0 += kInfGroup * L.sw) {
                            const uint32_t s = u % kInfRing, round = u / kInfRing;
                            if (u++ % kLoadWarps != lw) continue;
                            if (round > 0 && !mbar_wait(smem_u32(&sh->empty[s]), (round - 1) & 1u, abort)) continue;
                            const uint32_t bytes = static_cast<uint32_t>(L.npad) * min(kInfGroup * L.sw, L.kaug - g0) * 2u;
                            mbar_expect_tx(smem_u32(&sh->full[s]), bytes);
                            bulk_load(smem_u32(ring + s * kInfSlot), p.w_img + L.w_off + static_cast<int64_t>(L.npad) * g0 * 2,
                                      bytes, smem_u32(&sh->full[s]));
                        }
                    }
            }
        }
        cta_sync();
        if (tid == kLoadWarp * 32 && *abort && p.error) atomicExch(p.error, 1);
        return;
    }

    if (warp == kMmaWarp) {
        if (lane == 0) {
            // each tile's barriers complete once per (pair, layer): k counts those
            uint32_t u = 0, k = 0;
            for (int64_t pr = blockIdx.x; pr < n_pairs; pr += gridDim.x)
                for (int l = 0; l < NL; ++l, ++k)
                    for (int t = 0; t < 2; ++t) {
                        const LayerGeo& L = G.l[l];
                        // the tile's input for this layer is written (and its TMEM read)
                        mbar_wait(smem_u32(&sh->edone[t]), k & 1u, abort);
                        tc_after();
                        const uint32_t a0 = smem_u32(smem + t * kImgBytes);
                        const uint32_t sbo_a = static_cast<uint32_t>(L.kaug >> 3) << 7;
                        const uint32_t idesc = instr_desc(kRows, L.npad, false, false);
                        for (int g0 = 0; g0 < L.kaug; g0 += kInfGroup * L.sw) {
                            const uint32_t s = u % kInfRing, round = u / kInfRing;
                            ++u;
                            const bool ok = mbar_wait(smem_u32(&sh->full[s]), round & 1u, abort);
                            tc_after();
                            const uint32_t sb = smem_u32(ring + s * kInfSlot);
                            for (int k0 = g0; ok && k0 < min(g0 + kInfGroup * L.sw, L.kaug); k0 += L.sw) {
                                const int kw = min(L.sw, L.kaug - k0);
                                const uint32_t b0 = sb + static_cast<uint32_t>(L.npad * (k0 - g0) * 2);
                                const uint32_t sbo_b = static_cast<uint32_t>(kw >> 3) << 7;
                                for (int ks = 0; ks < (kw >> 4); ++ks)
                                    mma_bf16(tmem + static_cast<uint32_t>(t * 256),
                                             smem_desc(a0 + ((k0 >> 3) + 2 * ks) * 128u, 128u, sbo_a),
                                             smem_desc(b0 + ks * 256u, 128u, sbo_b), idesc, (k0 > 0 || ks > 0) ? 1u : 0u);
                            }
                            mma_commit(smem_u32(&sh->empty[s]));
                        }
                        mma_commit(smem_u32(&sh->mdone[t]));
                    }
        }
        __syncwarp();
    } else {
        // ---- epilogue warps: stage the first pair, then for every pair, layer and
        // tile in the MMA order: wait for the MMAs, apply GELU in place (or write the
        // logits and stage the tile of the next pair), arrive
        const int quarter = warp & 3, grp = warp >> 2;
        const int r = quarter * 32 + lane;
        uint32_t k = 0;  // (pair, layer) steps done
        const LayerGeo& L0 = G.l[0];
        const int64_t first = blockIdx.x;
        for (int t = 0; t < 2; ++t) {
            if (first < n_pairs) infer_stage(p, L0, smem + t * kImgBytes, (2 * first + t) * kRows, tid);
            proxy_fence();
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_u32(&sh->edone[t]));
        }
        for (int64_t pr = first; pr < n_pairs; pr += gridDim.x)
            for (int l = 0; l < NL; ++l, ++k)
                for (int t = 0; t < 2; ++t) {
                    const LayerGeo& L = G.l[l];
                    uint8_t* act = smem + t * kImgBytes;
                    const bool ok = __all_sync(0xffffffffu, mbar_wait(smem_u32(&sh->mdone[t]), k & 1u, abort));
                    tc_after();
                    const uint32_t tm = tmem + static_cast<uint32_t>(t * 256) + (static_cast<uint32_t>(quarter * 32) << 16);
                    const int64_t row = (2 * pr + t) * kRows + r;
                    if (l + 1 < NL) {
                        const LayerGeo& Ln = G.l[l + 1];
                        if (grp < L.n_pieces) {
                            const int pc = grp;
                            for (int cc = 0; ok && cc < L.ph[pc];) {
                                const int rem = L.ph[pc] - cc, col = L.p0[pc] + cc;
                                const uint32_t ta = tm + static_cast<uint32_t>(col);
                                // 64 columns per TMEM round trip where the piece has them
                                if (rem >= 64) {
                                    uint32_t v[64];
                                    tmem_ld64(ta, v);
                                    gelu_cols(v, act, Ln.kaug, r, col);
                                    cc += 64;
                                } else if (rem >= 32) {
                                    uint32_t v[32];
                                    tmem_ld32(ta, v);
                                    gelu_cols(v, act, Ln.kaug, r, col);
                                    cc += 32;
                                } else {
                                    uint32_t v[16];
                                    tmem_ld16(ta, v);
                                    gelu_cols(v, act, Ln.kaug, r, col);
                                    cc += 16;
                                }
                            }
                            if (pc == L.n_pieces - 1)
                                for (int col = L.dout; col < Ln.kaug; col += 8) {
                                    const uint32_t one = (row < p.n && col == L.dout) ? 0x3F80u : 0u;
                                    *reinterpret_cast<uint4*>(act + img_off(Ln.kaug, r, col)) = make_uint4(one, 0u, 0u, 0u);
                                }
                        }
                    } else {
                        if (grp == 0) {
                            uint32_t v[32];
                            if (ok) tmem_ld32(tm, v);
                            if (ok && row < p.n) {
                                float* o = p.logits + row * L.dout;
#pragma unroll
                                for (int c = 0; c < 32; ++c)
                                    if (c < L.dout) o[c] = __uint_as_float(v[c]);
                            }
                        }
                        const int64_t nxt = pr + gridDim.x;  // this tile of the next pair
                        if (nxt < n_pairs) infer_stage(p, L0, act, (2 * nxt + t) * kRows, tid);
                    }
                    proxy_fence();
                    tc_before();
                    __syncwarp();
                    if (lane == 0) mbar_arrive(smem_u32(&sh->edone[t]));
                }
    }
    tc_before();
    cta_sync();
    __syncwarp();
    if (tid == 0 && *abort && p.error) atomicExch(p.error, 1);
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512) : "memory");
}

// ---- weight gradients and AdamW ---------------------------------------------

struct DwTile {
    int layer, o0, oh, i0, iw;  // outputs [o0, o0 + oh) x inputs [i0, i0 + iw)
};

struct DwArgs {
    Geo geo;
    DwTile t[kMaxDwTiles];
    int n_tiles;
    int M;
    const uint8_t* scratch;
    uint8_t* w_img;
    float* w_aug;
    float* m1;
    float* m2;
    float* grad;  // non-null: write the summed gradient here, no AdamW
    float lr, b1, b2, eps, wd, bc1, bc2;
    int32_t* error;
};

struct DwSmem {
    uint64_t full[kDwStages], empty[kDwStages], done;
    uint32_t tmem;
    int abort;
};
static_assert(sizeof(DwSmem) <= kDwTail, "k_train_dw: barrier block");
static_assert(kDwSmem <= 227 * 1024, "k_train_dw: shared memory");
static_assert(kRows * (kDwMaxIn + 4) * 4 <= kDwStageBytes * kDwStages, "k_train_dw: the partial fits the stages");

// every thread of the cluster (non-aligned: warps may arrive diverged)
__device__ __forceinline__ void cluster_sync()
{
    asm volatile("barrier.cluster.arrive.release;\n\tbarrier.cluster.wait.acquire;" ::: "memory");
}

// four floats of CTA `rank`'s shared memory at the local address's offset
__device__ __forceinline__ float4 ld_cluster_v4(uint32_t local, uint32_t rank)
{
    uint32_t remote;
    float4 v;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(remote) : "r"(local), "r"(rank));
    asm volatile("ld.shared::cluster.v4.f32 {%0, %1, %2, %3}, [%4];"
                 : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
                 : "r"(remote)
                 : "memory");
    return v;
}

__device__ __forceinline__ float adamw_elem(float g, float* w, float* m1, float* m2, float wd, float lr, float b1,
                                            float b2, float eps, float bc1, float bc2)
{
    const float a = b1 * *m1 + (1.f - b1) * g;
    const float b = b2 * *m2 + (1.f - b2) * g * g;
    *m1 = a;
    *m2 = b;
    float x = *w * (1.f - lr * wd);
    x -= lr * (a / bc1) / (sqrtf(b / bc2) + eps);
    *w = x;
    return x;
}

// the BF16 images of augmented weight (o, i): the forward slab, and W^T for i < din
__device__ __forceinline__ void store_images(uint8_t* w_img, const LayerGeo& L, int layer, int o, int i, float x)
{
    const __nv_bfloat16 h = __float2bfloat16(x);
    *reinterpret_cast<__nv_bfloat16*>(w_img + L.w_off + w_elem(L, o, i)) = h;
    if (layer > 0 && i < L.din) *reinterpret_cast<__nv_bfloat16*>(w_img + L.wt_off + wt_elem(L, o, i)) = h;
}

__global__ void __launch_bounds__(kDwThreads, 1) k_train_dw(const __grid_constant__ DwArgs p)
{
    extern __shared__ __align__(1024) uint8_t smem[];
    DwSmem* sh = reinterpret_cast<DwSmem*>(smem + kDwStages * kDwStageBytes);
    volatile int* abort = &sh->abort;
    uint32_t rank, nrank;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(rank));
    asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(nrank));
    const DwTile T = p.t[blockIdx.x / nrank];
    const LayerGeo& L = p.geo.l[T.layer];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int tiles = (p.M + kRows - 1) / kRows;
    const int t0 = static_cast<int>(rank) * tiles / static_cast<int>(nrank);
    const int t1 = (static_cast<int>(rank) + 1) * tiles / static_cast<int>(nrank);
    const int nk = t1 - t0;
    const int iw = T.iw;
    const uint32_t ncol_b = static_cast<uint32_t>(iw >> 3) << 7;  // bytes of one row group of the staged inputs

    if (tid == 0) {
        for (int s = 0; s < kDwStages; ++s) {
            mbar_init(smem_u32(&sh->full[s]), kDwProducers);
            mbar_init(smem_u32(&sh->empty[s]), 1);
        }
        mbar_init(smem_u32(&sh->done), 1);
        sh->abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&sh->tmem)),
                     "r"(256)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (T.oh < kRows) {  // outputs past the tile read zeros (the copies fill only oh / 8 cores per row group)
        for (int s = 0; s < kDwStages; ++s)
            for (int i = tid; i < kDwABytes / 16; i += kDwThreads)
                reinterpret_cast<uint4*>(smem + s * kDwStageBytes)[i] = make_uint4(0u, 0u, 0u, 0u);
        proxy_fence();
    }
    tc_before();
    cta_sync();
    tc_after();
    const uint32_t tmem = sh->tmem;

    if (warp >= 1 && warp <= kDwProducers) {
        // ---- producers: per row tile, warp w takes row groups (w - 1) * G .. + G - 1
        // (G = 16 / kDwProducers): of the dZ image (the tile's outputs) by lanes
        // 0 .. G - 1, of the X image (the tile's inputs) by lanes G .. 2 G - 1
        constexpr int G = 16 / kDwProducers;
        for (int k = 0; k < nk; ++k) {
            const int s = k % kDwStages, round = k / kDwStages;
            bool ok = true;
            if (lane == 0 && round > 0) ok = mbar_wait(smem_u32(&sh->empty[s]), (round - 1) & 1, abort);
            ok = __shfl_sync(0xffffffffu, ok, 0);
            if (!ok) break;
            const uint32_t full = smem_u32(&sh->full[s]);
            if (lane == 0) mbar_expect_tx(full, static_cast<uint32_t>(T.oh + iw) * (kRows * 2) / kDwProducers);
            __syncwarp();
            const int t = t0 + k;
            const uint32_t a_s = smem_u32(smem + s * kDwStageBytes), b_s = a_s + kDwABytes;
            const int g = (warp - 1) * G + (lane % G);
            if (lane < G) {
                const uint32_t bytes = static_cast<uint32_t>(T.oh >> 3) << 7;
                bulk_load(a_s + g * 2048u,
                          p.scratch + L.z_off + static_cast<int64_t>(t) * L.z_tile +
                              (static_cast<int64_t>(g) * (L.npad >> 3) + (T.o0 >> 3)) * 128,
                          bytes, full);
            } else if (lane < 2 * G) {
                bulk_load(b_s + g * ncol_b,
                          p.scratch + L.x_off + static_cast<int64_t>(t) * L.x_tile +
                              (static_cast<int64_t>(g) * (L.kaug >> 3) + (T.i0 >> 3)) * 128,
                          ncol_b, full);
            }
        }
    } else if (warp == 0 && lane == 0) {
        // ---- MMAs: dW (outputs x inputs) += dZ^T X over the row tile, both operands MN-major
        const uint32_t idesc = instr_desc(kRows, iw, true, true);
        for (int k = 0; k < nk; ++k) {
            const int s = k % kDwStages, round = k / kDwStages;
            const bool ok = mbar_wait(smem_u32(&sh->full[s]), round & 1, abort);
            tc_after();
            const uint32_t a_s = smem_u32(smem + s * kDwStageBytes), b_s = a_s + kDwABytes;
            for (int ks = 0; ok && ks < kRows / 16; ++ks)
                mma_bf16(tmem, smem_desc(a_s + ks * 4096u, 2048u, 128u), smem_desc(b_s + ks * 2u * ncol_b, ncol_b, 128u),
                         idesc, (k > 0 || ks > 0) ? 1u : 0u);
            mma_commit(smem_u32(&sh->empty[s]));
        }
        if (nk > 0) mma_commit(smem_u32(&sh->done));
    }
    __syncwarp();

    // ---- this CTA's partial into its shared memory (FP32, rows of iw + 4)
    float* P = reinterpret_cast<float*>(smem);
    const int pitch = iw + 4;
    {
        const bool ok = __all_sync(0xffffffffu, nk > 0 && mbar_wait(smem_u32(&sh->done), 0, abort));
        tc_after();
        const int q = warp & 3, hh = warp >> 2;
        const int r = q * 32 + lane;
        for (int u = hh; u < (iw >> 4); u += kDwThreads / 128) {
            uint32_t v[16];
            if (ok) tmem_ld16(tmem + (static_cast<uint32_t>(q * 32) << 16) + static_cast<uint32_t>(u * 16), v);
            float4* d = reinterpret_cast<float4*>(P + r * pitch + u * 16);
#pragma unroll
            for (int j = 0; j < 4; ++j)
                d[j] = ok ? make_float4(__uint_as_float(v[4 * j]), __uint_as_float(v[4 * j + 1]),
                                        __uint_as_float(v[4 * j + 2]), __uint_as_float(v[4 * j + 3]))
                          : make_float4(0.f, 0.f, 0.f, 0.f);
        }
    }
    tc_before();
    cluster_sync();

    // ---- this CTA's share of the tile's rows: the partials of the cluster summed in
    // rank order, then the gradient out or the AdamW step
    {
        const int per = (T.oh + static_cast<int>(nrank) - 1) / static_cast<int>(nrank);
        const int rb = static_cast<int>(rank) * per, re = min(T.oh, rb + per);
        const uint32_t pbase = smem_u32(P);
        const int q4 = iw >> 2;  // groups of 4 columns
        for (int idx = tid; idx < (re - rb) * q4; idx += kDwThreads) {
            const int ol = rb + idx / q4, i = (idx % q4) * 4;
            const int o = T.o0 + ol;
            if (o >= L.dout || T.i0 + i > L.din) continue;
            const uint32_t la = pbase + static_cast<uint32_t>(ol * pitch + i) * 4u;
            float4 part[kMaxCluster];
#pragma unroll
            for (int q = 0; q < kMaxCluster; ++q)
                if (q < static_cast<int>(nrank)) part[q] = ld_cluster_v4(la, static_cast<uint32_t>(q));
            float4 g = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
            for (int q = 0; q < kMaxCluster; ++q)  // in rank order
                if (q < static_cast<int>(nrank)) {
                    g.x += part[q].x;
                    g.y += part[q].y;
                    g.z += part[q].z;
                    g.w += part[q].w;
                }
            // the 4 columns are consecutive in the row-major augmented arrays (16-byte
            // aligned: offsets, K_aug and the tile start are multiples of 4); columns
            // past the bias are padding, whose gradient is zero and which stay zero
            const int ia = T.i0 + i;
            const int64_t e = L.aug_off + static_cast<int64_t>(o) * L.kaug + ia;
            if (p.grad) {
                *reinterpret_cast<float4*>(p.grad + e) = g;
            } else {
                float4 w = *reinterpret_cast<const float4*>(p.w_aug + e);
                float4 a = *reinterpret_cast<const float4*>(p.m1 + e);
                float4 b = *reinterpret_cast<const float4*>(p.m2 + e);
                float* wv = &w.x;
                float* av = &a.x;
                float* bv = &b.x;
                const float gv[4] = {g.x, g.y, g.z, g.w};
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    adamw_elem(gv[j], wv + j, av + j, bv + j, ia + j < L.din ? p.wd : 0.f, p.lr, p.b1, p.b2, p.eps,
                               p.bc1, p.bc2);
                *reinterpret_cast<float4*>(p.w_aug + e) = w;
                *reinterpret_cast<float4*>(p.m1 + e) = a;
                *reinterpret_cast<float4*>(p.m2 + e) = b;
                // forward image: the 4 columns are 4 consecutive values of one core row
                const uint2 h = make_uint2(pack_bf16(w.x, w.y), pack_bf16(w.z, w.w));
                *reinterpret_cast<uint2*>(p.w_img + L.w_off + w_elem(L, o, ia)) = h;
                if (T.layer > 0) {
#pragma unroll
                    for (int j = 0; j < 4; ++j)
                        if (ia + j < L.din)
                            *reinterpret_cast<__nv_bfloat16*>(p.w_img + L.wt_off + wt_elem(L, o, ia + j)) =
                                __float2bfloat16(wv[j]);
                }
            }
        }
    }
    cluster_sync();
    if (tid == 0 && *abort && p.error) atomicExch(p.error, 1);
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(256) : "memory");
}

// ---- packing and the stand-alone AdamW (data parallel) ------------------------

struct GeoArgs {
    Geo geo;
};

__device__ __forceinline__ int layer_of(const Geo& G, int64_t e)
{
    int l = 0;
    while (l + 1 < G.n_layers && e >= G.l[l + 1].aug_off) ++l;
    return l;
}

__global__ void k_fused_pack(const __grid_constant__ GeoArgs a, const float* __restrict__ w_aug, uint8_t* w_img)
{
    const Geo& G = a.geo;
    for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < G.aug_elems;
         e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const LayerGeo& L = G.l[layer_of(G, e)];
        const int64_t el = e - L.aug_off;
        const int o = static_cast<int>(el / L.kaug), i = static_cast<int>(el - static_cast<int64_t>(o) * L.kaug);
        store_images(w_img, L, layer_of(G, e), o, i, w_aug[e]);
    }
}

struct AdamScalars {
    float lr, b1, b2, eps, wd, bc1, bc2;
};

__global__ void k_fused_adamw(const __grid_constant__ GeoArgs a, const AdamScalars h, float* w_aug, float* m1,
                              float* m2, const float* __restrict__ grad, uint8_t* w_img)
{
    const Geo& G = a.geo;
    for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < G.aug_elems;
         e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const LayerGeo& L = G.l[layer_of(G, e)];
        const int64_t el = e - L.aug_off;
        const int o = static_cast<int>(el / L.kaug), i = static_cast<int>(el - static_cast<int64_t>(o) * L.kaug);
        if (o >= L.dout || i > L.din) continue;
        const float x =
            adamw_elem(grad[e], w_aug + e, m1 + e, m2 + e, i < L.din ? h.wd : 0.f, h.lr, h.b1, h.b2, h.eps, h.bc1, h.bc2);
        store_images(w_img, L, layer_of(G, e), o, i, x);
    }
}

cudaError_t ensure_fused_smem()
{
    constexpr int kDevs = 64;
    static int done[kDevs];
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev >= 0 && dev < kDevs && __atomic_load_n(&done[dev], __ATOMIC_ACQUIRE)) return cudaSuccess;
    e = cudaFuncSetAttribute(k_train_fb, cudaFuncAttributeMaxDynamicSharedMemorySize, kFbSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_train_dw, cudaFuncAttributeMaxDynamicSharedMemorySize, kDwSmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_train_dw, cudaFuncAttributeNonPortableClusterSizeAllowed, 0);
    if (e == cudaSuccess && dev >= 0 && dev < kDevs) __atomic_store_n(&done[dev], 1, __ATOMIC_RELEASE);
    return e;
}

bool aligned16h(const void* ptr) { return (reinterpret_cast<uintptr_t>(ptr) & 15u) == 0; }

int grid_for(int64_t n)
{
    int64_t g = (n + 255) / 256;
    if (g > 148 * 8) g = 148 * 8;
    return static_cast<int>(g < 1 ? 1 : g);
}

}  // namespace

extern "C" {

int pb_train_fused_geometry(int32_t n_layers, const int32_t* dims, int32_t batch, int64_t* out, int32_t out_len)
{
    Geo g;
    const int rc = geo_build(n_layers, dims, batch, &g);
    if (rc != PB_SUCCESS) return rc;
    if (!out || out_len < 3 + 4 * n_layers) return PB_EINVAL;
    out[0] = g.img_bytes;
    out[1] = g.scratch_bytes;
    out[2] = g.aug_elems;
    for (int l = 0; l < n_layers; ++l) {
        out[3 + 4 * l + 0] = g.l[l].kaug;
        out[3 + 4 * l + 1] = g.l[l].npad;
        out[3 + 4 * l + 2] = g.l[l].aug_off;
        out[3 + 4 * l + 3] = g.l[l].w_off;
    }
    return PB_SUCCESS;
}

int pb_train_fused_pack(int32_t n_layers, const int32_t* dims, const float* w_aug, void* w_img, void* stream)
{
    GeoArgs a;
    const int rc = geo_build(n_layers, dims, 1, &a.geo);
    if (rc != PB_SUCCESS) return rc;
    if (!w_aug || !w_img || !aligned16h(w_img)) return PB_EINVAL;
    k_fused_pack<<<grid_for(a.geo.aug_elems), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        a, w_aug, static_cast<uint8_t*>(w_img));
    return cudaGetLastError() == cudaSuccess ? PB_SUCCESS : PB_ECUDA;
}

int pb_train_fused_step(int32_t n_layers, const int32_t* dims, const void* x_bf16, const int32_t* labels,
                        int32_t n_rows, const int32_t* rows, int32_t M, int32_t batch, float* w_aug, float* m1, float* m2,
                        void* w_img, void* scratch, float* grad, float lr, float beta1, float beta2, float eps,
                        float weight_decay, int32_t step, float* loss_sum, int32_t* correct, int32_t* error_flag,
                        void* stream)
{
    FbArgs* fb = new FbArgs();
    DwArgs* dw = new DwArgs();
    auto finish = [&](int rc) {
        delete fb;
        delete dw;
        return rc;
    };
    int rc = geo_build(n_layers, dims, batch, &fb->geo);
    if (rc != PB_SUCCESS) return finish(rc);
    if (M < 1 || M > batch || step < 1 || n_rows < 1) return finish(PB_EINVAL);
    if (!x_bf16 || !labels || !rows || !w_img || !scratch || !aligned16h(x_bf16) || !aligned16h(w_img) ||
        !aligned16h(scratch))
        return finish(PB_EINVAL);
    if (!grad && (!w_aug || !m1 || !m2)) return finish(PB_EINVAL);
    if (ensure_fused_smem() != cudaSuccess) return finish(PB_ECUDA);
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    fb->x = static_cast<const __nv_bfloat16*>(x_bf16);
    fb->labels = labels;
    fb->rows = rows;
    fb->n_rows = n_rows;
    fb->M = M;
    fb->scale = 1.f / static_cast<float>(M);
    fb->w_img = static_cast<const uint8_t*>(w_img);
    fb->scratch = static_cast<uint8_t*>(scratch);
    fb->loss_sum = loss_sum;
    fb->correct = correct;
    fb->error = error_flag;
    const int row_tiles = (M + kRows - 1) / kRows;
    k_train_fb<<<row_tiles, kFbThreads, kFbSmem, s>>>(*fb);
    if (cudaGetLastError() != cudaSuccess) return finish(PB_ECUDA);

    dw->geo = fb->geo;
    // weight tiles: 128 outputs x at most kDwMaxIn inputs (K_aug split evenly into
    // multiples of 16)
    int nt = 0;
    for (int l = 0; l < n_layers; ++l) {
        const LayerGeo& L = dw->geo.l[l];
        const int nr = (L.kaug + kDwMaxIn - 1) / kDwMaxIn;
        const int w0 = ((L.kaug + nr - 1) / nr + 15) / 16 * 16;
        for (int o0 = 0; o0 < L.npad; o0 += kRows)
            for (int i0 = 0; i0 < L.kaug; i0 += w0)
                dw->t[nt++] = DwTile{l, o0, min(kRows, L.npad - o0), i0, min(w0, L.kaug - i0)};
    }
    dw->n_tiles = nt;
    dw->M = M;
    dw->scratch = static_cast<const uint8_t*>(scratch);
    dw->w_img = static_cast<uint8_t*>(w_img);
    dw->w_aug = w_aug;
    dw->m1 = m1;
    dw->m2 = m2;
    dw->grad = grad;
    dw->lr = lr;
    dw->b1 = beta1;
    dw->b2 = beta2;
    dw->eps = eps;
    dw->wd = weight_decay;
    dw->bc1 = static_cast<float>(1.0 - std::pow(static_cast<double>(beta1), step));
    dw->bc2 = static_cast<float>(1.0 - std::pow(static_cast<double>(beta2), step));
    dw->error = error_flag;
    // the CTAs of a cluster split the row tiles: as many as fill the GPU once
    int cs = 148 / nt;
    cs = cs < 1 ? 1 : (cs > kMaxCluster ? kMaxCluster : cs);
    if (cs > row_tiles) cs = row_tiles;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(static_cast<unsigned>(nt * cs), 1, 1);
    cfg.blockDim = dim3(kDwThreads, 1, 1);
    cfg.dynamicSmemBytes = kDwSmem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = static_cast<unsigned>(cs);
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (cudaLaunchKernelEx(&cfg, k_train_dw, *dw) != cudaSuccess) return finish(PB_ECUDA);
    return finish(PB_SUCCESS);
}

int pb_mlp_infer_fused(int32_t n_layers, const int32_t* dims, const void* x_bf16, int64_t n, const void* w_img,
                       float* logits, int32_t* error_flag, void* stream)
{
    InferArgs a;
    const int rc = geo_build(n_layers, dims, 1, &a.geo);
    if (rc != PB_SUCCESS) return rc;
    if (n < 0 || !x_bf16 || !w_img || !logits || !aligned16h(x_bf16) || !aligned16h(w_img)) return PB_EINVAL;
    if (n == 0) return PB_SUCCESS;
    static int attr_done[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return PB_ECUDA;
    if (dev < 0 || dev >= 64 || !__atomic_load_n(&attr_done[dev], __ATOMIC_ACQUIRE)) {
        if (cudaFuncSetAttribute(k_mlp_infer_pp, cudaFuncAttributeMaxDynamicSharedMemorySize, kInfSmem) != cudaSuccess)
            return PB_ECUDA;
        if (dev >= 0 && dev < 64) __atomic_store_n(&attr_done[dev], 1, __ATOMIC_RELEASE);
    }
    a.x = static_cast<const __nv_bfloat16*>(x_bf16);
    a.n = n;
    a.w_img = static_cast<const uint8_t*>(w_img);
    a.logits = logits;
    a.error = error_flag;
    const int64_t pairs = ((n + kRows - 1) / kRows + 1) / 2;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const unsigned grid = static_cast<unsigned>(pairs < sms ? pairs : sms);
    k_mlp_infer_pp<<<grid, kFbThreads, kInfSmem, static_cast<cudaStream_t>(stream)>>>(a);
    return cudaGetLastError() == cudaSuccess ? PB_SUCCESS : PB_ECUDA;
}

int pb_train_fused_adamw(int32_t n_layers, const int32_t* dims, float* w_aug, float* m1, float* m2, const float* grad,
                         void* w_img, float lr, float beta1, float beta2, float eps, float weight_decay, int32_t step,
                         void* stream)
{
    GeoArgs a;
    const int rc = geo_build(n_layers, dims, 1, &a.geo);
    if (rc != PB_SUCCESS) return rc;
    if (!w_aug || !m1 || !m2 || !grad || !w_img || !aligned16h(w_img) || step < 1) return PB_EINVAL;
    AdamScalars h{lr, beta1, beta2, eps, weight_decay,
                  static_cast<float>(1.0 - std::pow(static_cast<double>(beta1), step)),
                  static_cast<float>(1.0 - std::pow(static_cast<double>(beta2), step))};
    k_fused_adamw<<<grid_for(a.geo.aug_elems), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        a, h, w_aug, m1, m2, grad, static_cast<uint8_t*>(w_img));
    return cudaGetLastError() == cudaSuccess ? PB_SUCCESS : PB_ECUDA;
}

}  // extern "C"
