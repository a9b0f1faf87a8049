// Layout of the caller-provided scratch buffer of pb_solve_batch (host and device).
//
//   [feature windows] n_traj x n_window_columns x window floats (PB_FEAT_IS_WINDOW kinds)
//   [step records]    n_traj x cap x record_stride bytes        (PB_DENSE_DEFERRED)
//   [tails]           n_traj x tail_stride bytes                (PB_DENSE_DEFERRED)
//   [split save grid] n_save x (float hi, float lo)            (PB_DENSE_DEFERRED)
//   [saved states]    n_traj x state_stride bytes               (PB_SCHED_PROBED)
//   [sort keys/values] 4 x n_traj int32                         (PB_SCHED_PROBED)
//   [drain]           2 x u64 counters, n_traj int32 published ids, n_traj u8
//                     sampled flags                              (PB_SCHED_PROBED)
//   [radix-sort temporary storage]                               (PB_SCHED_PROBED; its
//                     size is added on the host)
//
// Each part starts on a 256-byte boundary.  A step record (a multiple of 16 bytes,
// written with 16-byte stores) is
//   double t, double dt, int32 first_save, int32 n_saves,
//   for each statistics state: y, h*k1, c, b, a   (stage precision), padding
// and a tail is
//   int32 n_records (-1 = capacity exceeded), int32 next_save, int32 status, int32 pad,
//   double fill[dim]   (value of the save points after the last record)
#pragma once
#include "pb_compat.cuh"

#include "pybasin_b200.h"

namespace pb {

constexpr int PB_MAX_STAT_STATES = 8;
// record header: t (f64), dt (f64), first covered save index, number of covered
// saves (i32 each); the statistics slots follow
constexpr int kRecordHeader = 24;
constexpr int kRecordIndexOffset = 16;
constexpr int kDefaultRecordCap = 1024;

struct ScratchLayout {
    int64_t median_off;
    int64_t rec_off;
    int64_t tail_off;
    int64_t state_off;     // PB_SCHED_PROBED: integrator state saved after the probe phase
    int64_t key_in_off;    // probe-phase step counts, in queue order
    int64_t key_out_off;
    int64_t val_in_off;    // trajectory ids, in queue order
    int64_t val_out_off;   // trajectory ids, longest predicted first
    int64_t drain_off;     // main phase sampling drained into the integrator (probed): two
                           // u64 counters (published, claimed), then the published
                           // trajectory ids + 1 (int32, n_traj), then sampled flags (u8, n_traj)
    int64_t sort_tmp_off;  // radix-sort temporary storage (last)
    int64_t split_off;     // deferred dense output: (hi, lo) float split of the save grid
    int64_t total;         // excluding the radix-sort temporary
    int32_t rec_stride;
    int32_t cap;
    int32_t tail_stride;
    int32_t deferred;
    int32_t state_stride;
    int32_t probed;
};

// Bytes of one saved integrator state: y, yc, k1 (stage precision), then t, dt,
// next save time (double) and si, steps, status, n_records, done (int32).
__host__ __device__ constexpr int saved_state_bytes(int dim, int rsize)
{
    return ((3 * dim * rsize + 7) / 8 * 8 + 3 * 8 + 5 * 4 + 15) / 16 * 16;
}

__host__ __device__ inline int64_t align_up(int64_t v, int64_t a) { return (v + a - 1) / a * a; }

// columns whose feature needs the stored window (median, quantiles, moments, ...)
__host__ __device__ inline int count_median_columns(const pb_solve_args& a)
{
    int m = 0;
    for (int c = 0; c < a.n_features; ++c) m += PB_FEAT_IS_WINDOW(a.feat_kind[c]) ? 1 : 0;
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
        l.rec_stride = static_cast<int32_t>(align_up(kRecordHeader + 5 * count_stat_states(a) * rsize, 16));
        int64_t cap = a.window_record_cap > 0 ? a.window_record_cap : kDefaultRecordCap;
        if (cap > nwin) cap = nwin;
        l.cap = static_cast<int32_t>(cap);
        l.rec_off = off;
        off = align_up(off + a.n_traj * cap * l.rec_stride, 256);
        l.tail_stride = static_cast<int32_t>(align_up(16 + 8 * a.dim, 16));
        l.tail_off = off;
        off = align_up(off + a.n_traj * l.tail_stride, 256);
        l.split_off = off;
        off = align_up(off + static_cast<int64_t>(a.n_save) * 8, 256);
        l.probed = (a.schedule == PB_SCHED_PROBED) ? 1 : 0;
        if (l.probed) {
            l.state_stride = saved_state_bytes(a.dim, rsize);
            l.state_off = off;
            off = align_up(off + a.n_traj * l.state_stride, 256);
            const int64_t vec = align_up(a.n_traj * 4, 256);
            l.key_in_off = off;
            l.key_out_off = off + vec;
            l.val_in_off = off + 2 * vec;
            l.val_out_off = off + 3 * vec;
            off += 4 * vec;
            l.drain_off = off;
            off += 256 + vec + align_up(a.n_traj, 256);
            l.sort_tmp_off = off;
        }
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

__device__ __forceinline__ unsigned char* state_ptr(const pb_solve_args& a, const ScratchLayout& l, int64_t traj)
{
    return static_cast<unsigned char*>(a.scratch) + l.state_off + traj * l.state_stride;
}
// drain region of the probed schedule (see ScratchLayout::drain_off)
__host__ __device__ inline int64_t drain_bytes(const ScratchLayout& l, int64_t n_traj)
{
    return l.probed ? 256 + align_up(n_traj * 4, 256) + align_up(n_traj, 256) : 0;
}
__device__ __forceinline__ unsigned long long* drain_counters(const pb_solve_args& a, const ScratchLayout& l)
{
    return reinterpret_cast<unsigned long long*>(static_cast<unsigned char*>(a.scratch) + l.drain_off);
}
__device__ __forceinline__ int* drain_list(const pb_solve_args& a, const ScratchLayout& l)
{
    return reinterpret_cast<int*>(static_cast<unsigned char*>(a.scratch) + l.drain_off + 256);
}
__device__ __forceinline__ unsigned char* drain_sampled(const pb_solve_args& a, const ScratchLayout& l, int64_t n)
{
    return static_cast<unsigned char*>(a.scratch) + l.drain_off + 256 + align_up(n * 4, 256);
}

__device__ __forceinline__ unsigned* sort_vec(const pb_solve_args& a, int64_t off)
{
    return reinterpret_cast<unsigned*>(static_cast<unsigned char*>(a.scratch) + off);
}

}  // namespace pb
