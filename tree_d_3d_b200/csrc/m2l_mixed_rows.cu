// Mixed-precision M2L of the log kernel on the CUDA cores, a group of 8 lanes per
// destination row (the FP32 counterpart of fmm_m2l_host, K/fmm_m2l_host/
// fmm_m2l_host_pyccel.py:16-105, on size-scaled expansions).
//
// Layout: every source cell is one packed record (td3_pack_m2l_sources): its centre in
// FP64, its moments scaled by its size, hat_k = a_k / h^k, in FP32 pairs, and h / unit,
// 8 (P + 4) bytes (128 bytes at P = 12: one cache line per gathered partner).
//
// Work: a warp owns a run of whole destination rows (an even share of the entries, each
// row counting 8 more).
// Its four 8-lane groups take the rows in order, each row whole: lane i of a group
// translates entries i, i + 8, ... of the row and adds the contributions into its own
// FP32 sums, kept in shared memory (a warp's sums column-major with a 33-word stride: a
// column's accesses hit 32 banks, freeing registers for more resident warps); at the
// row's end lane i sums columns i, i + 8, ... over the group's 8 lanes pairwise and adds
// them to the FP64 locals.  Rows longer than LONG_ROW entries are taken by the whole
// warp first (32 partial rows), so no group holds a warp for long.  Every destination
// is summed by one group in a fixed order: deterministic results.
#include "common.cuh"

namespace {

constexpr int RW = 4;          // warps per block
constexpr int GL = 8;          // lanes per destination group
constexpr int LONG_ROW = 96;   // rows longer than this are taken by the whole warp
constexpr int ROW_COST = GL;   // entries a row counts for in the warps' shares
constexpr unsigned FULL = 0xffffffffu;
constexpr int MAX_DEVICES = 64;

template <int P>
struct RowCoef {
    float c[(P + 1) * (P + 1)];
};

// float4 words of a packed source record of template order P (W = P + 1 odd, so
// 16 + 8 W + 8 bytes is a whole number of 16-byte words).
template <int P>
constexpr int rec_words() {
    return (P + 4) / 2;
}

int rec_order(int order) { return order <= 4 ? 4 : order <= 8 ? 8 : order <= 12 ? 12 : order <= 16 ? 16 : 20; }

// Record word q of node `node`: word 0 the centre (two doubles); words 1.. the scaled
// moment pairs (k, k + 1) for k = 2 (q - 1), the pair k = W being (h / unit, 0).
template <int P>
__global__ void k_pack_m2l_sources(i64 count, int order, const double* __restrict__ mre,
                                   const double* __restrict__ mim,
                                   const double* __restrict__ center,
                                   const double* __restrict__ half, double inv_unit,
                                   float4* __restrict__ rec) {
    td3_chain_wait();
    td3_chain_release();
    constexpr int W = P + 1, F4 = rec_words<P>();
    i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count * F4) return;
    i64 node = t / F4;
    int q = (int)(t % F4);
    if (q == 0) {
        double2 c = reinterpret_cast<const double2*>(center)[node];
        rec[t] = *reinterpret_cast<float4*>(&c);
        return;
    }
    int w = order + 1;
    double h = half[node], inv = 1.0 / h;
    float v[4];
#pragma unroll
    for (int j = 0; j < 2; ++j) {
        int k = 2 * (q - 1) + j;
        float re = 0.0f, im = 0.0f;
        if (k < w) {
            // a_k / h^k by repeated division, as td3_scale_moments
            double s = 1.0;
            for (int i = 0; i < k; ++i) s *= inv;
            re = (float)(mre[node * w + k] * s);
            im = (float)(mim[node * w + k] * s);
        } else if (k == W) {
            re = (float)(h * inv_unit);
        }
        v[2 * j] = re;
        v[2 * j + 1] = im;
    }
    rec[t] = make_float4(v[0], v[1], v[2], v[3]);
}

// The packed record of source `src` (16-byte loads through the read-only path).
template <int P>
__device__ __forceinline__ void load_record(const float4* __restrict__ rec, i64 src,
                                            float4 (&m)[rec_words<P>()]) {
    const float4* r = rec + src * rec_words<P>();
#pragma unroll
    for (int q = 0; q < rec_words<P>(); ++q) m[q] = __ldg(r + q);
}

// One translation from the source whose record is `m` into this lane's sums `acc`
// (columns 2l, 2l + 1: bhat_l in units of the destination size; 2W, 2W + 1: a_0).
template <int P, class Acc>
__device__ __forceinline__ void translate(const float4 (&m)[rec_words<P>()], double cx, double cy,
                                          float fhd, double inv_unit, const RowCoef<P>& C,
                                          Acc& acc) {
    constexpr int W = P + 1, F4 = rec_words<P>();
    const double2 c = *reinterpret_cast<const double2*>(&m[0]);
    float hr[W + 1], hi[W + 1];
#pragma unroll
    for (int q = 1; q < F4; ++q) {
        hr[2 * q - 2] = m[q].x;
        hi[2 * q - 2] = m[q].y;
        hr[2 * q - 1] = m[q].z;
        hi[2 * q - 1] = m[q].w;
    }
    const float fhs = hr[W];
    // t = c_dst - c_src in FP64, then in units of `unit` in FP32
    const float fr = (float)((cx - c.x) * inv_unit), fi = (float)((cy - c.y) * inv_unit);
    const float t2 = fr * fr + fi * fi;
    const float inv = __fdividef(1.0f, t2);
    const float ur = fr * inv, ui = -fi * inv;  // unit / t
    const float wsr = fhs * ur, wsi = fhs * ui;  // h_src / t
    const float wdr = fhd * ur, wdi = fhd * ui;  // h_dst / t
    const float lnt = 0.5f * __logf(t2);         // ln |t / unit|
    float ar[W], ai[W];
    float pr = 1.0f, pi = 0.0f;
#pragma unroll
    for (int k = 0; k < W; ++k) {
        ar[k] = hr[k] * pr - hi[k] * pi;
        ai[k] = hr[k] * pi + hi[k] * pr;
        const float nr = pr * wsr - pi * wsi;
        pi = pr * wsi + pi * wsr;
        pr = nr;
    }
    float qr = wdr, qi = wdi;
#pragma unroll
    for (int l = 0; l < W; ++l) {
        float sr = 0.0f, si = 0.0f;
#pragma unroll
        for (int k = 0; k < W; ++k) {
            sr = fmaf(C.c[k * W + l], ar[k], sr);
            si = fmaf(C.c[k * W + l], ai[k], si);
        }
        if (l == 0) {
            acc[0] += fmaf(ar[0], lnt, -sr);
            acc[1] += fmaf(ai[0], lnt, -si);
        } else {
            // bhat_l = -(-1)^l s_l wd^l
            const float sg = (l & 1) ? 1.0f : -1.0f;
            acc[2 * l] = fmaf(sg * sr, qr, acc[2 * l]);
            acc[2 * l] = fmaf(-sg * si, qi, acc[2 * l]);
            acc[2 * l + 1] = fmaf(sg * sr, qi, acc[2 * l + 1]);
            acc[2 * l + 1] = fmaf(sg * si, qr, acc[2 * l + 1]);
            const float nr = qr * wdr - qi * wdi;
            qi = qr * wdi + qi * wdr;
            qr = nr;
        }
    }
    acc[2 * W] += ar[0];
    acc[2 * W + 1] += ai[0];
}

// A lane's partial sums in shared memory: column c of lane L at c * 33 + L (a warp's
// accesses of one column hit 32 banks; a group's 8 lanes of a column are contiguous).
struct SmemAcc {
    float* base;  // the warp's array plus the lane
    __device__ __forceinline__ float& operator[](int c) const { return base[c * 33]; }
};

// Sum of column c over the lanes [8 g0, 8 g0 + 8 G) of a warp's SmemAcc array, pairwise
// in a fixed order.
template <int G>
__device__ __forceinline__ float smem_column_sum(const float* a, int c, int g0) {
    float gs[G];
#pragma unroll
    for (int g = 0; g < G; ++g) {
        const float* p = a + c * 33 + 8 * (g0 + g);
        gs[g] = ((p[0] + p[1]) + (p[2] + p[3])) + ((p[4] + p[5]) + (p[6] + p[7]));
    }
    if (G == 1) return gs[0];
    return (gs[0] + gs[G > 1 ? 1 : 0]) + (gs[G > 2 ? 2 : 0] + gs[G > 3 ? 3 : 0]);
}

template <int P>
__global__ void __launch_bounds__(32 * RW)
k_m2l_mixed_rows(const i64* __restrict__ row_start, const i64* __restrict__ partners, i64 n_dst,
                 const double* __restrict__ dst_center, const double* __restrict__ dst_half,
                 const float4* __restrict__ rec, int order, const RowCoef<P> C, double unit,
                 double* __restrict__ local_re, double* __restrict__ local_im) {
    td3_chain_wait();
    td3_chain_release();
    constexpr int W = P + 1, V = 2 * W + 2;
    __shared__ float accs[RW][V * 33];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5, g = lane >> 3, gl = lane & 7;
    float* wacc = accs[wib];
    const int w = order + 1;
    const double inv_unit = 1.0 / unit, ln_unit = log(unit);
    // this warp's rows [da, db): an even share of the cost entries + ROW_COST x rows (a
    // row takes a group at least one round, however few its entries: a run of empty or
    // short rows must not fall to one warp)
    const i64 gw = (i64)blockIdx.x * RW + wib, nw = (i64)gridDim.x * RW;
    const i64 total = row_start[n_dst] + ROW_COST * n_dst, share = (total + nw - 1) / nw;
    auto first_row_at = [&](i64 e) {
        i64 lo = 0, hi = n_dst;
        while (lo < hi) {
            i64 mid = (lo + hi) >> 1;
            if (row_start[mid] + ROW_COST * mid < e) lo = mid + 1;
            else hi = mid;
        }
        return lo;
    };
    const i64 da = first_row_at(gw * share);
    const i64 db = gw + 1 == nw ? n_dst : first_row_at((gw + 1) * share);
    if (da >= db) return;
    // this lane's partial sums (shared memory, 72 registers per thread instead of 96)
    SmemAcc acc{wacc + lane};
#pragma unroll
    for (int c = 0; c < V; ++c) acc[c] = 0.0f;

    // 1. rows longer than LONG_ROW: the whole warp, 32 entries per round
    for (i64 base = da; base < db; base += 32) {
        const i64 dl = base + lane;
        const bool is_long = dl < db && row_start[dl + 1] - row_start[dl] > LONG_ROW;
        unsigned longs = __ballot_sync(FULL, is_long);
        while (longs) {
            const i64 d = base + (__ffs(longs) - 1);
            longs &= longs - 1;
            const double cx = dst_center[2 * d], cy = dst_center[2 * d + 1], hd = dst_half[d];
            const float fhd = (float)(hd * inv_unit);
            const i64 e1 = row_start[d + 1];
            for (i64 e = row_start[d] + lane; e < e1; e += 32) {
                float4 m[rec_words<P>()];
                load_record<P>(rec, partners[e], m);
                translate<P>(m, cx, cy, fhd, inv_unit, C, acc);
            }
            __syncwarp();
            if (lane < 2 * W && (lane >> 1) < w) {
                const int l = lane >> 1;
                double sc = 1.0;
                const double inv_h = 1.0 / hd;
                for (int i = 0; i < l; ++i) sc *= inv_h;
                double add = (double)smem_column_sum<4>(wacc, lane, 0) * sc;
                if (lane < 2) add += ln_unit * (double)smem_column_sum<4>(wacc, 2 * W + lane, 0);
                ((lane & 1) ? local_im : local_re)[d * w + l] += add;
            }
            __syncwarp();
#pragma unroll
            for (int c = 0; c < V; ++c) acc[c] = 0.0f;
            __syncwarp();
        }
    }

    // 2. the other rows: a group per row, the groups taking the rows in order
    i64 next = da + 4;
    i64 d = da + g < db ? da + g : -1;
    i64 cur = 0, end = 0;
    double cx = 0.0, cy = 0.0;
    float fhd = 0.0f;
    auto claim = [&]() {
        if (d < 0) return;
        cur = row_start[d];
        end = row_start[d + 1];
        if (end - cur > LONG_ROW) end = cur;  // done in part 1
        cx = dst_center[2 * d];
        cy = dst_center[2 * d + 1];
        fhd = (float)(dst_half[d] * inv_unit);
    };
    claim();
    bool had = end > cur;
    while (__any_sync(FULL, d >= 0)) {
        const i64 e = cur + gl;
        const i64 src = d >= 0 && e < end ? partners[e] : -1;
        if (src >= 0) {
            float4 m[rec_words<P>()];
            load_record<P>(rec, src, m);
            translate<P>(m, cx, cy, fhd, inv_unit, C, acc);
        }
        cur += GL;
        const bool done = d >= 0 && cur >= end;
        const unsigned dm = __ballot_sync(FULL, done);
        if (!dm) continue;
        __syncwarp();
        if (done && had) {
            // lane gl adds columns gl + 8 j (coefficient l = gl / 2 + 4 j) to the locals
            const double inv_h = 1.0 / dst_half[d];
            double sc = 1.0, h4 = inv_h * inv_h;
            h4 *= h4;
            for (int i = 0; i < (gl >> 1); ++i) sc *= inv_h;
#pragma unroll
            for (int j = 0; j < (2 * W + 7) / 8; ++j) {
                const int c = gl + 8 * j, l = c >> 1;
                if (c < 2 * W && l < w) {
                    double add = (double)smem_column_sum<1>(wacc, c, g) * sc;
                    if (c < 2) add += ln_unit * (double)smem_column_sum<1>(wacc, 2 * W + c, g);
                    ((c & 1) ? local_im : local_re)[d * w + l] += add;
                }
                sc *= h4;
            }
        }
        __syncwarp();
        if (done) {
#pragma unroll
            for (int c = 0; c < V; ++c) acc[c] = 0.0f;
        }
        // the finished groups take the next rows, in group order
        const unsigned gm = dm & 0x01010101u;
        const int rank = __popc(gm & ((1u << (8 * g)) - 1u));
        if (done) {
            d = next + rank < db ? next + rank : -1;
            claim();
            had = end > cur;
        }
        next += __popc(gm);
    }
}

template <int P>
int launch_rows(const i64* row_start, const i64* partners, i64 n_dst, const double* dst_center,
                const double* dst_half, const float* rec, int order, const double* coeff,
                double unit, double* lre, double* lim, cudaStream_t s) {
    RowCoef<P> C;
    const int w = order + 1;
    for (int k = 0; k <= P; ++k)
        for (int l = 0; l <= P; ++l)
            C.c[k * (P + 1) + l] = (k < w && l < w) ? (float)coeff[k * w + l] : 0.0f;
    // one resident wave of blocks, each warp an even share of the entries
    // (the per-device figures are cached; concurrent first calls store the same values)
    static int per_sm[MAX_DEVICES] = {};
    static int sms[MAX_DEVICES] = {};
    int dev = 0;
    TD3_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= MAX_DEVICES) return TD3_EINVAL;
    if (!per_sm[dev]) {
        int n = 0, b = 0;
        TD3_TRY(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
        TD3_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_m2l_mixed_rows<P>, 32 * RW, 0));
        sms[dev] = n;
        per_sm[dev] = b > 0 ? b : 1;
    }
    i64 blocks = (i64)sms[dev] * per_sm[dev];
    const i64 max_blocks = (n_dst + RW - 1) / RW;
    if (blocks > max_blocks) blocks = max_blocks;
    TD3_TRY(td3_launch_chained(k_m2l_mixed_rows<P>, (unsigned)blocks, 32 * RW, 0, s, row_start,
                               partners, n_dst, dst_center, dst_half,
                               reinterpret_cast<const float4*>(rec), order, C, unit, lre, lim));
    TD3_CHECK_LAUNCH();
    return TD3_OK;
}

template <int P>
int launch_pack(i64 count, int order, const double* mre, const double* mim, const double* center,
                const double* half, double unit, float* rec, cudaStream_t s) {
    const i64 threads = count * rec_words<P>();
    TD3_TRY(td3_launch_chained(k_pack_m2l_sources<P>, td3_blocks(threads, 256), 256, 0, s, count,
                               order, mre, mim, center, half, 1.0 / unit,
                               reinterpret_cast<float4*>(rec)));
    TD3_CHECK_LAUNCH();
    return TD3_OK;
}

}  // namespace

extern "C" int td3_m2l_record_floats(int order) {
    if (order < 0 || order > 20) return TD3_EINVAL;
    return 4 * ((rec_order(order) + 4) / 2);
}

extern "C" int td3_pack_m2l_sources(int64_t count, int order, const double* moment_re,
                                    const double* moment_im, const double* node_center,
                                    const double* node_half, double unit, float* records,
                                    void* stream) {
    if (count < 0 || order < 0 || order > 20) return TD3_EINVAL;
    if (!(unit > 0.0 && unit < INFINITY)) return TD3_EINVAL;
    if (count == 0) return TD3_OK;
    cudaStream_t s = td3_stream(stream);
    switch (rec_order(order)) {
        case 4: return launch_pack<4>(count, order, moment_re, moment_im, node_center, node_half, unit, records, s);
        case 8: return launch_pack<8>(count, order, moment_re, moment_im, node_center, node_half, unit, records, s);
        case 12: return launch_pack<12>(count, order, moment_re, moment_im, node_center, node_half, unit, records, s);
        case 16: return launch_pack<16>(count, order, moment_re, moment_im, node_center, node_half, unit, records, s);
        default: return launch_pack<20>(count, order, moment_re, moment_im, node_center, node_half, unit, records, s);
    }
}

extern "C" int td3_fmm_m2l_mixed_rows(const int64_t* row_start, const int64_t* partners,
                                      int64_t n_dst, const double* dst_center,
                                      const double* dst_half, const float* records, int order,
                                      const double* coeff, double unit, double* local_re,
                                      double* local_im, void* stream) {
    if (n_dst < 0 || order < 0 || order > 20) return TD3_EINVAL;
    if (!(unit > 0.0 && unit < INFINITY)) return TD3_EINVAL;
    if (n_dst == 0) return TD3_OK;
    cudaStream_t s = td3_stream(stream);
    switch (rec_order(order)) {
        case 4: return launch_rows<4>(row_start, partners, n_dst, dst_center, dst_half, records, order, coeff, unit, local_re, local_im, s);
        case 8: return launch_rows<8>(row_start, partners, n_dst, dst_center, dst_half, records, order, coeff, unit, local_re, local_im, s);
        case 12: return launch_rows<12>(row_start, partners, n_dst, dst_center, dst_half, records, order, coeff, unit, local_re, local_im, s);
        case 16: return launch_rows<16>(row_start, partners, n_dst, dst_center, dst_half, records, order, coeff, unit, local_re, local_im, s);
        default: return launch_rows<20>(row_start, partners, n_dst, dst_center, dst_half, records, order, coeff, unit, local_re, local_im, s);
    }
}
