// Z-order (Morton) keys of the initial conditions: the processing order that
// keeps neighbouring ICs (which mostly share an attractor and a step count) in
// the same warp.  Two kernels: a bounding-box reduction over the first
// min(dim, 4) coordinates and the key computation.  The arithmetic is the
// FP64 formula of pybasin_b200.engine.spatial_order (same operations in the same
// order), so the keys are bit-identical to it on finite inputs.
#include <cuda_runtime.h>

#include <cstdint>

#include <cub/device/device_radix_sort.cuh>

#include "pybasin_b200.h"

namespace pb {

constexpr int kMaxMortonDims = 4;

// order-preserving map of a double onto uint64 (for atomicMin / atomicMax)
__device__ __forceinline__ unsigned long long ordered_bits(double x)
{
    const unsigned long long b = static_cast<unsigned long long>(__double_as_longlong(x));
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double from_ordered_bits(unsigned long long u)
{
    const unsigned long long b = (u >> 63) ? (u & 0x7fffffffffffffffull) : ~u;
    return __longlong_as_double(static_cast<long long>(b));
}

template <class T>
__global__ void __launch_bounds__(256) k_bbox(const T* __restrict__ y0, int64_t n, int dim, int d,
                                              unsigned long long* __restrict__ box)
{
    unsigned long long mn[kMaxMortonDims], mx[kMaxMortonDims];
#pragma unroll
    for (int k = 0; k < kMaxMortonDims; ++k) {
        mn[k] = ~0ull;
        mx[k] = 0ull;
    }
    const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
#pragma unroll
        for (int k = 0; k < kMaxMortonDims; ++k) {
            if (k >= d) break;
            const double x = static_cast<double>(y0[i * dim + k]);
            if (x != x) continue;  // NaN coordinates do not widen the box
            const unsigned long long u = ordered_bits(x);
            mn[k] = min(mn[k], u);
            mx[k] = max(mx[k], u);
        }
    }
#pragma unroll
    for (int k = 0; k < kMaxMortonDims; ++k) {
        for (int o = 16; o > 0; o >>= 1) {
            mn[k] = min(mn[k], __shfl_xor_sync(0xffffffffu, mn[k], o));
            mx[k] = max(mx[k], __shfl_xor_sync(0xffffffffu, mx[k], o));
        }
    }
    if ((threadIdx.x & 31) == 0) {
#pragma unroll
        for (int k = 0; k < kMaxMortonDims; ++k) {
            if (k >= d) break;
            atomicMin(box + k, mn[k]);
            atomicMax(box + kMaxMortonDims + k, mx[k]);
        }
    }
}

template <class T>
__global__ void __launch_bounds__(256) k_morton(const T* __restrict__ y0, int64_t n, int dim, int d, int bits,
                                                const int32_t* __restrict__ groups,
                                                const unsigned long long* __restrict__ box,
                                                int64_t* __restrict__ keys)
{
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double top = static_cast<double>((1ll << bits) - 1);
    unsigned long long key = 0ull;
    for (int k = 0; k < d; ++k) {
        const double lo = box[k] == ~0ull ? 0.0 : from_ordered_bits(box[k]);
        const double hi = box[k] == ~0ull ? 0.0 : from_ordered_bits(box[kMaxMortonDims + k]);
        const double span = fmax(hi - lo, 1e-300);
        double v = (static_cast<double>(y0[i * dim + k]) - lo) / span * top;
        if (v != v) v = 0.0;
        v = fmin(fmax(v, 0.0), top);
        const unsigned long long q = static_cast<unsigned long long>(static_cast<long long>(v));
        unsigned long long spread = 0ull;
        for (int b = 0; b < bits; ++b) spread |= ((q >> b) & 1ull) << (b * d);
        key |= spread << k;
    }
    if (groups) {
        const int shift = bits * d > 40 ? bits * d - 40 : 0;
        key = (static_cast<unsigned long long>(static_cast<long long>(groups[i])) << 40) | (key >> shift);
    }
    keys[i] = static_cast<long long>(key);
}

__global__ void k_iota(int32_t* __restrict__ v, int64_t n)
{
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) v[i] = static_cast<int32_t>(i);
}

// scratch of pb_morton_order: alternate key buffer, alternate index buffer, then
// the radix sort's temporary storage, each 256-byte aligned
struct SortScratch {
    size_t keys_alt, vals_alt, temp, temp_bytes, total;
};

inline size_t align256(size_t v) { return (v + 255) / 256 * 256; }

inline bool sort_scratch(int64_t n, SortScratch& l)
{
    l.temp_bytes = 0;
    cub::DoubleBuffer<unsigned long long> k(nullptr, nullptr);
    cub::DoubleBuffer<int32_t> v(nullptr, nullptr);
    if (cub::DeviceRadixSort::SortPairs(nullptr, l.temp_bytes, k, v, static_cast<int>(n)) != cudaSuccess)
        return false;
    l.keys_alt = 0;
    l.vals_alt = align256(static_cast<size_t>(n) * sizeof(unsigned long long));
    l.temp = l.vals_alt + align256(static_cast<size_t>(n) * sizeof(int32_t));
    l.total = l.temp + align256(l.temp_bytes);
    return true;
}

}  // namespace pb

using namespace pb;

extern "C" int64_t pb_morton_order_scratch_bytes(int64_t n)
{
    if (n < 0 || n > 0x7fffffffLL) return -1;
    SortScratch l;
    if (!sort_scratch(n < 1 ? 1 : n, l)) return -1;
    return static_cast<int64_t>(l.total);
}

extern "C" int pb_morton_order(int64_t* keys, int64_t n, int32_t end_bit, void* scratch, int64_t scratch_bytes,
                               int32_t* order_out, void* stream)
{
    if (n < 0 || n > 0x7fffffffLL || end_bit < 1 || end_bit > 64) return PB_EINVAL;
    if (n == 0) return PB_SUCCESS;
    if (!keys || !scratch || !order_out) return PB_EINVAL;
    SortScratch l;
    if (!sort_scratch(n, l)) return PB_ECUDA;
    if (scratch_bytes < static_cast<int64_t>(l.total)) return PB_EINVAL;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    unsigned char* b = static_cast<unsigned char*>(scratch);
    k_iota<<<static_cast<unsigned>((n + 255) / 256), 256, 0, st>>>(order_out, n);
    cub::DoubleBuffer<unsigned long long> k(reinterpret_cast<unsigned long long*>(keys),
                                            reinterpret_cast<unsigned long long*>(b + l.keys_alt));
    cub::DoubleBuffer<int32_t> v(order_out, reinterpret_cast<int32_t*>(b + l.vals_alt));
    size_t tb = l.temp_bytes;
    if (cub::DeviceRadixSort::SortPairs(b + l.temp, tb, k, v, static_cast<int>(n), 0, end_bit, st) != cudaSuccess)
        return PB_ECUDA;
    if (v.Current() != order_out &&
        cudaMemcpyAsync(order_out, v.Current(), static_cast<size_t>(n) * sizeof(int32_t), cudaMemcpyDeviceToDevice,
                        st) != cudaSuccess)
        return PB_ECUDA;
    return cudaGetLastError() == cudaSuccess ? PB_SUCCESS : PB_ECUDA;
}

extern "C" int pb_morton_keys(const void* y0, int32_t y0_dtype, int64_t n, int32_t dim, int32_t bits,
                              const int32_t* groups, uint64_t* bbox_work, int64_t* keys_out, void* stream)
{
    if (n < 0 || dim <= 0) return PB_EINVAL;
    if (n == 0) return PB_SUCCESS;
    if (!y0 || !bbox_work || !keys_out) return PB_EINVAL;
    if (y0_dtype != PB_DTYPE_F32 && y0_dtype != PB_DTYPE_F64) return PB_EINVAL;
    const int d = dim < kMaxMortonDims ? dim : kMaxMortonDims;
    if (bits < 1 || bits * d > 62) return PB_EINVAL;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // box[0..3] = min (identity all ones), box[4..7] = max (identity zero)
    cudaError_t e = cudaMemsetAsync(bbox_work, 0xff, kMaxMortonDims * sizeof(uint64_t), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(bbox_work + kMaxMortonDims, 0, kMaxMortonDims * sizeof(uint64_t), st);
    if (e != cudaSuccess) return PB_ECUDA;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return PB_ECUDA;
    const int64_t need = (n + 255) / 256;
    const unsigned rblocks = static_cast<unsigned>(need < 4LL * sms ? need : 4LL * sms);
    const int64_t kblocks = need;
    if (kblocks > 0x7fffffffLL) return PB_EINVAL;
    auto box = reinterpret_cast<unsigned long long*>(bbox_work);
    if (y0_dtype == PB_DTYPE_F32) {
        auto p = static_cast<const float*>(y0);
        k_bbox<float><<<rblocks, 256, 0, st>>>(p, n, dim, d, box);
        k_morton<float><<<static_cast<unsigned>(kblocks), 256, 0, st>>>(p, n, dim, d, bits, groups, box, keys_out);
    } else {
        auto p = static_cast<const double*>(y0);
        k_bbox<double><<<rblocks, 256, 0, st>>>(p, n, dim, d, box);
        k_morton<double><<<static_cast<unsigned>(kblocks), 256, 0, st>>>(p, n, dim, d, bits, groups, box, keys_out);
    }
    return cudaGetLastError() == cudaSuccess ? PB_SUCCESS : PB_ECUDA;
}
