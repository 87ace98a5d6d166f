// Device pieces shared by the mixed-precision M2L kernels that walk the CSR entries of
// the M2L rows 32 at a time (one translation per lane), whatever the destinations.
//
// A warp owns a run of whole rows (an even share of the entries, cut at row boundaries)
// and takes their entries in rounds of 32.  A round can hold several destinations: the
// lanes of one destination are summed by a segmented scan (fixed order), the last lane
// of each destination adds the sums to its FP64 locals, and a destination that goes on
// into the next round hands its partial sums to that round's lane 0 through shared
// memory.  Each destination is written once, by one warp: deterministic results.
#pragma once

#include "common.cuh"

namespace td3m2l {

// The first d in [0, n) with row_start[d] >= e (n if none).
__device__ __forceinline__ i64 first_row_at(const i64* __restrict__ row_start, i64 n, i64 e) {
    i64 lo = 0, hi = n;
    while (lo < hi) {
        i64 mid = (lo + hi) >> 1;
        if (row_start[mid] < e) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// The entries [e0, e1) of warp `gw` of `nw`: an even share, cut at row boundaries.
__device__ __forceinline__ void warp_entries(const i64* __restrict__ row_start, i64 n_dst, i64 gw,
                                             i64 nw, i64& e0, i64& e1) {
    i64 total = row_start[n_dst];
    i64 share = (total + nw - 1) / nw;
    i64 da = first_row_at(row_start, n_dst, gw * share);
    i64 db = gw + 1 == nw ? n_dst : first_row_at(row_start, n_dst, (gw + 1) * share);
    e0 = row_start[da];
    e1 = row_start[db];
}

// Inclusive segmented sum over the lanes: lanes with equal `key` (contiguous runs)
// are summed, the last lane of a run ending with the run's total.
template <int V>
__device__ __forceinline__ void segmented_scan(float (&v)[V], int key, int lane) {
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        int k = __shfl_up_sync(0xffffffffu, key, off);
        bool take = lane >= off && k == key;
#pragma unroll
        for (int j = 0; j < V; ++j) {
            float y = __shfl_up_sync(0xffffffffu, v[j], off);
            if (take) v[j] += y;
        }
    }
}

// local_l += b_l / h^l for l < w (b_l = (v[2l], v[2l+1])), plus ln(unit) times the
// source charge sums (v[2W], v[2W+1]) for l = 0.
template <int W>
__device__ __forceinline__ void add_locals(const float (&v)[2 * W + 2], i64 d, int w,
                                           const double* __restrict__ dst_half, double ln_unit,
                                           double* __restrict__ local_re,
                                           double* __restrict__ local_im) {
    double inv_h = 1.0 / dst_half[d], scale = 1.0;
#pragma unroll
    for (int l = 0; l < W; ++l) {
        if (l < w) {
            double ur = l ? 0.0 : ln_unit * (double)v[2 * W];
            double ui = l ? 0.0 : ln_unit * (double)v[2 * W + 1];
            local_re[d * w + l] += (double)v[2 * l] * scale + ur;
            local_im[d * w + l] += (double)v[2 * l + 1] * scale + ui;
        }
        scale *= inv_h;
    }
}

// After the contributions of a round are in v (lane order = entry order): sum each
// destination's lanes, add finished destinations to the locals, and hand a destination
// that continues in the next round to that round's lane 0 (carry, carry_d).
template <int W>
__device__ __forceinline__ void finish_round(float (&v)[2 * W + 2], int d, bool live, int lane,
                                             i64 next_e, i64 e1, const int* __restrict__ entry_row,
                                             int w, const double* __restrict__ dst_half,
                                             double ln_unit, double* __restrict__ local_re,
                                             double* __restrict__ local_im, float* carry,
                                             int& carry_d) {
    constexpr int V = 2 * W + 2;
    if (lane == 0 && live && d == carry_d) {
#pragma unroll
        for (int j = 0; j < V; ++j) v[j] += carry[j];
    }
    segmented_scan<V>(v, d, lane);
    int d_next = __shfl_down_sync(0xffffffffu, d, 1);
    int d_last = __shfl_sync(0xffffffffu, d, 31);
    bool cont = next_e < e1 && entry_row[next_e] == d_last;
    bool last = live && (lane == 31 ? !cont : d_next != d);
    if (last) add_locals<W>(v, d, w, dst_half, ln_unit, local_re, local_im);
    __syncwarp();
    if (lane == 31 && cont) {
#pragma unroll
        for (int j = 0; j < V; ++j) carry[j] = v[j];
    }
    carry_d = cont ? d_last : -1;
    __syncwarp();
}

}  // namespace td3m2l
