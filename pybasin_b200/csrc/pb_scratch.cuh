// Layout of the caller-provided scratch buffer of pb_solve_batch (host and device).
//
//   [median windows]  n_traj x n_median_columns x window floats (PB_FEAT_MEDIAN)
//   [step records]    n_traj x cap x record_stride bytes        (PB_DENSE_DEFERRED)
//   [tails]           n_traj x tail_stride bytes                (PB_DENSE_DEFERRED)
//
// Each part starts on a 256-byte boundary.  A step record (a multiple of 16 bytes,
// written with 16-byte stores) is
//   double t, double 1/dt,
//   for each statistics state: y, h*k1, c, b, a   (stage precision),
//   int32 first_save, int32 n_saves, padding
// and a tail is
//   int32 n_records (-1 = capacity exceeded), int32 next_save, int32 status, int32 pad,
//   double fill[dim]   (value of the save points after the last record)
#pragma once
#include <stdint.h>

#include "pybasin_b200.h"

namespace pb {

constexpr int PB_MAX_STAT_STATES = 8;
constexpr int kRecordHeader = 16;  // t, 1/dt
constexpr int kDefaultRecordCap = 1024;

struct ScratchLayout {
    int64_t median_off;
    int64_t rec_off;
    int64_t tail_off;
    int64_t total;
    int32_t rec_stride;
    int32_t cap;
    int32_t tail_stride;
    int32_t deferred;
};

__host__ __device__ inline int64_t align_up(int64_t v, int64_t a) { return (v + a - 1) / a * a; }

__host__ __device__ inline int count_median_columns(const pb_solve_args& a)
{
    int m = 0;
    for (int c = 0; c < a.n_features; ++c) m += (a.feat_kind[c] == PB_FEAT_MEDIAN);
    return m;
}

__host__ __device__ inline int count_stat_states(const pb_solve_args& a)
{
    unsigned mask = 0;
    for (int c = 0; c < a.n_features; ++c)
        if (a.feat_state[c] >= 0 && a.feat_state[c] < 32) mask |= 1u << a.feat_state[c];
    int n = 0;
    for (int s = 0; s < 32; ++s) n += (mask >> s) & 1u;
    return n;
}

__host__ __device__ inline ScratchLayout scratch_layout(const pb_solve_args& a)
{
    ScratchLayout l{};
    const int64_t nwin = a.n_save - a.win_begin;
    int64_t off = 0;
    l.median_off = 0;
    off = align_up(a.n_traj * count_median_columns(a) * nwin * static_cast<int64_t>(sizeof(float)), 256);
    const bool network = a.system == PB_SYS_ROSSLER_NET;  // features from the final state, no windows
    if (network) {
        l.total = 0;
        return l;
    }
    l.deferred = (a.dense_mode == PB_DENSE_DEFERRED && a.n_features > 0 && a.y_full_out == nullptr) ? 1 : 0;
    if (l.deferred) {
        const int rsize = a.precision == PB_PREC_FP64 ? 8 : 4;
        l.rec_stride = static_cast<int32_t>(align_up(kRecordHeader + 5 * count_stat_states(a) * rsize + 8, 16));
        int64_t cap = a.window_record_cap > 0 ? a.window_record_cap : kDefaultRecordCap;
        if (cap > nwin) cap = nwin;
        l.cap = static_cast<int32_t>(cap);
        l.rec_off = off;
        off = align_up(off + a.n_traj * cap * l.rec_stride, 256);
        l.tail_stride = static_cast<int32_t>(align_up(16 + 8 * a.dim, 16));
        l.tail_off = off;
        off = align_up(off + a.n_traj * l.tail_stride, 256);
    }
    l.total = off;
    return l;
}

__device__ __forceinline__ float* median_ptr(const pb_solve_args& a, const ScratchLayout& l)
{
    return reinterpret_cast<float*>(static_cast<unsigned char*>(a.scratch) + l.median_off);
}
__device__ __forceinline__ unsigned char* record_ptr(const pb_solve_args& a, const ScratchLayout& l, int64_t traj,
                                                     int k)
{
    return static_cast<unsigned char*>(a.scratch) + l.rec_off + (traj * l.cap + k) * l.rec_stride;
}
__device__ __forceinline__ unsigned char* tail_ptr(const pb_solve_args& a, const ScratchLayout& l, int64_t traj)
{
    return static_cast<unsigned char*>(a.scratch) + l.tail_off + traj * l.tail_stride;
}

// offset of (first_save, n_saves) inside a record
__host__ __device__ inline int record_index_offset(int ns, int rsize) { return kRecordHeader + 5 * ns * rsize; }

}  // namespace pb
