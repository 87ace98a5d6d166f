// The mixed-precision M2L of the log kernel with its matrix products on the tensor
// cores (tcgen05.mma, kind tf32, 3xTF32), for orders up to 15.  The arithmetic is that
// of the FP32 form (fmm_log.cu, k_m2l_mixed), which follows fmm_m2l_host
// (K/fmm_m2l_host/fmm_m2l_host_pyccel.py:16-105) on size-scaled expansions:
//   a'_k = hat_k ws^k,  s_l = sum_k coeff[k, l] a'_k,
//   b_0 += a_0 ln|t / L| - s_0 (+ ln L a_0 in FP64),  b_l += -(-1)^l s_l wd^l,
//   local_l += b_l / h_dst^l (FP64).
// A CTA is 4 warps; each warp owns a run of whole rows and walks their entries 32 at a
// time (m2l_rows.cuh), one translation per lane, as its quarter of a 128-row tile.
// Per tile:
//   1. lane r of warp w forms a'_k as row 32 w + r of A (128 x 32: real parts in columns
//      0-15, imaginary parts in 16-31), each value split into its TF32 rounding and the
//      TF32 rounding of the remainder (hi + lo);
//   2. one thread issues D = A_hi B_hi^T + A_hi B_lo^T + A_lo B_hi^T (M = 128, N = 32,
//      K = 32 as four steps of 8) with B the reference's matrix twice on the block
//      diagonal (row n = l, column k), FP32 accumulation in tensor memory, completion on
//      an mbarrier;
//   3. each lane reads its row of D (tcgen05.ld: warp w reads lanes 32 w..32 w + 31),
//      forms its contributions b_l, and the warp sums them per destination (segmented
//      scan in lane order) into the FP64 locals.
// A warp that has finished its rows feeds zero rows until the CTA's last tile.
#include "common.cuh"
#include "tcgen05.cuh"
#include "m2l_rows.cuh"

namespace {

constexpr int TC_THREADS = 128;
constexpr int TC_K = 32;                  // 16 real + 16 imaginary columns
constexpr int TC_N = 32;
constexpr int TC_LBO = 128;               // bytes between core matrices along K
constexpr int TC_SBO = (TC_K / 4) * 128;  // bytes between groups of 8 rows
constexpr int TC_A_BYTES = TC_THREADS * TC_K * 4;
constexpr int TC_B_BYTES = TC_N * TC_K * 4;
constexpr int TC_BLOCKS_PER_SM = 5;
constexpr uint32_t TC_WAIT_LIMIT = 1u << 24;

template <int P>
struct TcCoef {
    float c[(P + 1) * (P + 1)];
};

// Byte offset of element (row, k) in the K-major, unswizzled operand layout.
__device__ __forceinline__ int tc_offset(int row, int k) {
    return (row >> 3) * TC_SBO + (k >> 2) * TC_LBO + (row & 7) * 16 + (k & 3) * 4;
}

template <int P>
__global__ void __launch_bounds__(TC_THREADS)
k_m2l_tc(const i64* __restrict__ row_start, const int* __restrict__ entry_row,
         const i64* __restrict__ partners, i64 n_dst, const double* __restrict__ dst_center,
         const double* __restrict__ dst_half, const double* __restrict__ src_center,
         const double* __restrict__ src_half, const float2* __restrict__ hat, int order,
         const TcCoef<P> C, double unit, double* __restrict__ local_re,
         double* __restrict__ local_im, i64* status) {
    constexpr int W = P + 1, V = 2 * W + 2;
    static_assert(W <= 16, "orders up to 15");
    __shared__ __align__(1024) unsigned char sA[2][TC_A_BYTES];  // hi, lo
    __shared__ __align__(1024) unsigned char sB[2][TC_B_BYTES];
    __shared__ float carry[TC_THREADS / 32][V];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tmem_base;
    const int r = threadIdx.x, lane = r & 31, warp = r >> 5;
    const int w = order + 1;

    // B: coeff twice on the block diagonal, split into TF32 hi and lo
    for (int i = r; i < TC_N * TC_K; i += TC_THREADS) {
        int n = i / TC_K, k = i % TC_K;
        float v = 0.0f;
        if ((n < 16) == (k < 16)) {
            int l = n & 15, kk = k & 15;
            if (l < W && kk < W) v = C.c[kk * W + l];
        }
        float hi = td3tc::to_tf32(v);
        *reinterpret_cast<float*>(sB[0] + tc_offset(n, k)) = hi;
        *reinterpret_cast<float*>(sB[1] + tc_offset(n, k)) = td3tc::to_tf32(v - hi);
    }
    if (r == 0) td3tc::mbar_init(&bar, 1);
    if (warp == 0) td3tc::tmem_alloc(&tmem_base, 32);
    td3tc::fence_smem_for_async();
    td3tc::fence_before_sync();
    __syncthreads();
    td3tc::fence_after_sync();
    const uint32_t tmem = tmem_base;

    i64 base, e1;
    td3m2l::warp_entries(row_start, n_dst, (i64)blockIdx.x * (TC_THREADS / 32) + warp,
                         (i64)gridDim.x * (TC_THREADS / 32), base, e1);
    double inv_unit2 = 1.0 / (unit * unit), ln_unit = log(unit);
    int carry_d = -1;
    uint32_t phase = 0;
    bool failed = false;
    for (;; base += 32) {
        bool has = base < e1;
        if (!__syncthreads_or(has)) break;
        // 1. this lane's row of A
        i64 e = base + lane;
        bool live = has && e < e1;
        int d = live ? entry_row[e] : -1;
        float wdr = 0.0f, wdi = 0.0f, lnt = 0.0f;
        float ar[W], ai[W];
#pragma unroll
        for (int k = 0; k < W; ++k) ar[k] = ai[k] = 0.0f;
        if (live) {
            i64 src = partners[e];
            double cx = dst_center[2 * d], cy = dst_center[2 * d + 1], hd = dst_half[d];
            double tr = cx - src_center[2 * src], ti = cy - src_center[2 * src + 1];
            double t2 = tr * tr + ti * ti, inv = 1.0 / t2, hs = src_half[src];
            float wsr = (float)(hs * tr * inv), wsi = (float)(-hs * ti * inv);
            wdr = (float)(hd * tr * inv);
            wdi = (float)(-hd * ti * inv);
            lnt = 0.5f * log_split(t2 * inv_unit2);
            const float2* a = hat + src * td3_hat_width(order);
            float hr[W + 1], hi[W + 1];
#pragma unroll
            for (int c = 0; c < (W + 1) / 2; ++c) {
                float4 m = td3_hat_pair(a, c, w);
                hr[2 * c] = m.x;
                hi[2 * c] = m.y;
                hr[2 * c + 1] = m.z;
                hi[2 * c + 1] = m.w;
            }
            float pr = 1.0f, pi = 0.0f;
#pragma unroll
            for (int k = 0; k < W; ++k) {
                float2 m = make_float2(hr[k], hi[k]);
                ar[k] = m.x * pr - m.y * pi;
                ai[k] = m.x * pi + m.y * pr;
                float nr = pr * wsr - pi * wsi;
                pi = pr * wsi + pi * wsr;
                pr = nr;
            }
        }
#pragma unroll
        for (int c = 0; c < TC_K / 4; ++c) {
            float hi[4], lo[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                int k = 4 * c + j, kk = k & 15;
                float v = kk < W ? (k < 16 ? ar[kk] : ai[kk]) : 0.0f;
                hi[j] = td3tc::to_tf32(v);
                lo[j] = td3tc::to_tf32(v - hi[j]);
            }
            *reinterpret_cast<float4*>(sA[0] + tc_offset(r, 4 * c)) =
                make_float4(hi[0], hi[1], hi[2], hi[3]);
            *reinterpret_cast<float4*>(sA[1] + tc_offset(r, 4 * c)) =
                make_float4(lo[0], lo[1], lo[2], lo[3]);
        }
        // every warp has read the previous tile's rows of D before this barrier
        td3tc::fence_smem_for_async();
        td3tc::fence_before_sync();
        __syncthreads();
        td3tc::fence_after_sync();
        // 2. the products
        if (r == 0) {
            constexpr uint32_t idesc = td3tc::idesc_tf32(TC_THREADS, TC_N);
            const int pa[3] = {0, 0, 1}, pb[3] = {0, 1, 0};
            uint32_t acc = 0;
#pragma unroll
            for (int p = 0; p < 3; ++p)
#pragma unroll
                for (int ks = 0; ks < TC_K / 8; ++ks) {
                    uint64_t da = td3tc::smem_desc(td3tc::smem_addr(sA[pa[p]]) + 2 * TC_LBO * ks,
                                                   TC_LBO, TC_SBO);
                    uint64_t db = td3tc::smem_desc(td3tc::smem_addr(sB[pb[p]]) + 2 * TC_LBO * ks,
                                                   TC_LBO, TC_SBO);
                    td3tc::mma_tf32(tmem, da, db, idesc, acc);
                    acc = 1;
                }
            td3tc::mma_commit(&bar);
        }
        bool ok = td3tc::mbar_wait(&bar, phase, TC_WAIT_LIMIT);
        phase ^= 1u;
        if (!__syncthreads_and(ok)) {  // one decision for the whole block
            failed = true;
            if (r == 0) td3_report(status, 1);
            break;
        }
        td3tc::fence_after_sync();
        // 3. this lane's row of D: s_l real in columns 0-15, imaginary in 16-31
        float s[32];
        td3tc::tmem_load32(tmem + ((uint32_t)(32 * warp) << 16), s);
        float v[V];
#pragma unroll
        for (int j = 0; j < V; ++j) v[j] = 0.0f;
        if (live) {
            v[0] = ar[0] * lnt - s[0];
            v[1] = ai[0] * lnt - s[16];
            float qr = wdr, qi = wdi;
#pragma unroll
            for (int l = 1; l < W; ++l) {
                float sign = (l & 1) ? 1.0f : -1.0f;
                float sr = s[l], si = s[16 + l];
                v[2 * l] = sign * (sr * qr - si * qi);
                v[2 * l + 1] = sign * (sr * qi + si * qr);
                float nr = qr * wdr - qi * wdi;
                qi = qr * wdi + qi * wdr;
                qr = nr;
            }
            v[2 * W] = ar[0];
            v[2 * W + 1] = ai[0];
        }
        if (has)
            td3m2l::finish_round<W>(v, d, live, lane, base + 32, e1, entry_row, w, dst_half,
                                    ln_unit, local_re, local_im, carry[warp], carry_d);
    }
    if (failed) td3tc::mbar_wait(&bar, phase ^ 1u, TC_WAIT_LIMIT);  // products still in flight
    td3tc::fence_before_sync();
    __syncthreads();
    td3tc::fence_after_sync();
    if (warp == 0) td3tc::tmem_free(tmem, 32);
}

template <int P>
int launch(const i64* row_start, const int* entry_row, const i64* partners, i64 n_dst, const double* dst_center,
           const double* dst_half, const double* src_center, const double* src_half,
           const float2* hat, int order, const double* coeff, double unit, double* lre,
           double* lim, i64* status, cudaStream_t s) {
    TcCoef<P> C;
    int w = order + 1;
    for (int k = 0; k <= P; ++k)
        for (int l = 0; l <= P; ++l)
            C.c[k * (P + 1) + l] = (k < w && l < w) ? (float)coeff[k * w + l] : 0.0f;
    int device = 0, sms = 148;
    TD3_TRY(cudaGetDevice(&device));
    TD3_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    k_m2l_tc<P><<<sms * TC_BLOCKS_PER_SM, TC_THREADS, 0, s>>>(
        row_start, entry_row, partners, n_dst, dst_center, dst_half, src_center, src_half, hat,
        order, C, unit, lre, lim, status);
    TD3_CHECK_LAUNCH();
    return TD3_OK;
}

}  // namespace

int td3_m2l_tensor(const i64* row_start, const int* entry_row, const i64* partners, i64 n_dst, const double* dst_center,
                   const double* dst_half, const double* src_center, const double* src_half,
                   const float2* hat, int order, const double* coeff, double unit,
                   double* local_re, double* local_im, i64* status, cudaStream_t s) {
    if (order <= 4)
        return launch<4>(row_start, entry_row, partners, n_dst, dst_center, dst_half, src_center, src_half,
                         hat, order, coeff, unit, local_re, local_im, status, s);
    if (order <= 8)
        return launch<8>(row_start, entry_row, partners, n_dst, dst_center, dst_half, src_center, src_half,
                         hat, order, coeff, unit, local_re, local_im, status, s);
    if (order <= 12)
        return launch<12>(row_start, entry_row, partners, n_dst, dst_center, dst_half, src_center, src_half,
                          hat, order, coeff, unit, local_re, local_im, status, s);
    return launch<15>(row_start, entry_row, partners, n_dst, dst_center, dst_half, src_center, src_half, hat,
                      order, coeff, unit, local_re, local_im, status, s);
}
