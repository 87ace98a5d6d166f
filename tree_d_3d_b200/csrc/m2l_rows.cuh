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

// The column form of a round's sums: the round's contributions (v, lane order = entry
// order) are staged in shared memory (`stage`, 32 x (2W + 2) floats of this warp), then
// lane k sums column k (and k + 32, ...) over the round's entries in order, carrying the
// destination that continues into the next round in `col` (compensated sums: `comp` holds
// each one's running error), and at each destination's last entry the sums go to its
// FP64 locals (b_l = bhat_l / h^l, plus ln(unit) times the source charge sums for l = 0):
// a coalesced write per destination, and no shuffle per value.  Each destination belongs
// to one warp: deterministic sums.
template <int W>
__device__ __forceinline__ void column_round(const float (&v)[2 * W + 2], int d, bool live,
                                             int lane, i64 next_e, i64 e1,
                                             const int* __restrict__ entry_row, int w,
                                             const double* __restrict__ dst_half, double ln_unit,
                                             double* __restrict__ local_re,
                                             double* __restrict__ local_im, float* stage,
                                             float (&col)[(2 * W + 2 + 31) / 32],
                                             float (&comp)[(2 * W + 2 + 31) / 32]) {
    constexpr int V = 2 * W + 2, NC = (V + 31) / 32;
    static_assert(V % 4 == 0, "rows of whole float4s");
#pragma unroll
    for (int c = 0; c < V / 4; ++c)
        reinterpret_cast<float4*>(stage + lane * V)[c] =
            make_float4(v[4 * c], v[4 * c + 1], v[4 * c + 2], v[4 * c + 3]);
    // lane i ends its destination's entries unless entry i + 1 (or the next round's first)
    // has the same destination
    const int d_next = __shfl_down_sync(0xffffffffu, d, 1);
    const bool cont = next_e < e1 && entry_row[next_e] == __shfl_sync(0xffffffffu, d, 31);
    const unsigned ends = __ballot_sync(0xffffffffu, live && (lane == 31 ? !cont : d_next != d));
    const unsigned lives = __ballot_sync(0xffffffffu, live);
    __syncwarp();
    for (int i = 0; i < 32 && ((lives >> i) & 1u); ++i) {
        // compensated (Kahan) sums: the error of a destination's sum stays at a few
        // roundings whatever its length
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            if (lane + 32 * c < V) {
                const float y = stage[i * V + lane + 32 * c] - comp[c];
                const float t = col[c] + y;
                comp[c] = (t - col[c]) - y;
                col[c] = t;
            }
        }
        if ((ends >> i) & 1u) {
            const int di = __shfl_sync(0xffffffffu, d, i);
            // the source charge sums (columns 2W, 2W + 1) to lanes 0 and 1
            const float a0 = __shfl_sync(0xffffffffu, col[(2 * W) / 32] - comp[(2 * W) / 32],
                                         ((2 * W) & 31) + (lane & 1));
            const double inv_h = 1.0 / dst_half[di];
#pragma unroll
            for (int c = 0; c < NC; ++c) {
                const int k = lane + 32 * c, l = k >> 1;
                if (k < 2 * W && l < w) {
                    double scale = 1.0;
                    for (int t = 0; t < l; ++t) scale *= inv_h;
                    double add = ((double)col[c] - (double)comp[c]) * scale;
                    if (k < 2) add += ln_unit * (double)a0;
                    double* out = (k & 1) ? local_im : local_re;
                    out[(i64)di * w + l] += add;
                }
                col[c] = 0.0f;
                comp[c] = 0.0f;
            }
        }
    }
    __syncwarp();
}

}  // namespace td3m2l
