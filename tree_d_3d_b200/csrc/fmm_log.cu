// The FMM of the line-charge (log) kernel in complex form (Greengard-Rokhlin), FP64:
//   M2L by destination row    (K/fmm_m2l_host/fmm_m2l_host_pyccel.py:16-105; GPU form
//                              K/fmm_m2l/fmm_m2l_cuda.cu:12-80)
//   L2L per level             (K/fmm_downward/fmm_downward_pyccel.py:15-64)
//
// M2L: one warp per destination cell; the warp splits into groups of G lanes, lane l
// of a group owning expansion coefficient l (and l + G), each group taking every
// (32/G)-th partner; the scaled moments a'_k = a_k w^k pass through shared memory and
// s_l = sum_k coeff[k, l] a'_k is the real matrix product of the reference.  The
// partial locals of the groups are summed by shuffles and added once per cell.
#include "common.cuh"
#include "m2l_rows.cuh"

namespace {

constexpr int M2L_WARPS = 4;

template <int G, int CPL>
__global__ void __launch_bounds__(32 * M2L_WARPS)
k_m2l_log(const i64* __restrict__ row_start, const i64* __restrict__ partners, i64 n_dst,
          const double* __restrict__ dst_center, const double* __restrict__ src_center,
          const double* __restrict__ moment_re, const double* __restrict__ moment_im, int order,
          const double* __restrict__ coeff_g, double* __restrict__ local_re,
          double* __restrict__ local_im) {
    constexpr int GROUPS = 32 / G;
    constexpr int WMAX = G * CPL;
    constexpr int WC = WMAX < TD3_MAX_ORDER + 1 ? WMAX : TD3_MAX_ORDER + 1;
    __shared__ double coeff[WC * WC];
    __shared__ double2 abuf[M2L_WARPS][GROUPS][WMAX];
    int w = order + 1;
    for (int k = threadIdx.x; k < w * w; k += blockDim.x) coeff[k] = coeff_g[k];
    __syncthreads();
    int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    int g = lane / G, li = lane % G;
    for (i64 dst = (i64)blockIdx.x * M2L_WARPS + wib; dst < n_dst; dst += (i64)gridDim.x * M2L_WARPS) {
        i64 e0 = row_start[dst], e1 = row_start[dst + 1];
        if (e0 == e1) continue;
        double cx = dst_center[2 * dst], cy = dst_center[2 * dst + 1];
        double b_re[CPL], b_im[CPL];
#pragma unroll
        for (int j = 0; j < CPL; ++j) b_re[j] = b_im[j] = 0.0;
        // the groups walk the row in lockstep; a group past the end idles
        for (i64 base = e0; base < e1; base += GROUPS) {
            i64 e = base + g;
            bool live = e < e1;
            double pw_re[CPL], pw_im[CPL];
            double t_re = 0.0, t_im = 0.0, t2 = 1.0;
            i64 src = 0;
            if (live) {
                src = partners[e];
                t_re = cx - src_center[2 * src];
                t_im = cy - src_center[2 * src + 1];
                t2 = t_re * t_re + t_im * t_im;
                double inv = 1.0 / t2;
                double w_re = t_re * inv, w_im = -t_im * inv;
                // w^l by the reference's recurrence pw[k] = pw[k-1] * w
                double p_re = 1.0, p_im = 0.0;
                int k = 0;
#pragma unroll
                for (int j = 0; j < CPL; ++j) {
                    int l = li + j * G;
                    for (; k < l; ++k) {
                        double nr = p_re * w_re - p_im * w_im;
                        p_im = p_re * w_im + p_im * w_re;
                        p_re = nr;
                    }
                    pw_re[j] = p_re;
                    pw_im[j] = p_im;
                    double a_re = 0.0, a_im = 0.0;
                    if (l < w) {
                        a_re = moment_re[src * w + l];
                        a_im = moment_im[src * w + l];
                    }
                    abuf[wib][g][l] = make_double2(a_re * p_re - a_im * p_im, a_re * p_im + a_im * p_re);
                }
            }
            __syncwarp();
            if (live) {
#pragma unroll
                for (int j = 0; j < CPL; ++j) {
                    int l = li + j * G;
                    if (l >= w) continue;
                    double s_re = 0.0, s_im = 0.0;
                    for (int k = 0; k < w; ++k) {
                        double c = coeff[k * w + l];
                        double2 a = abuf[wib][g][k];
                        s_re += c * a.x;
                        s_im += c * a.y;
                    }
                    if (l == 0) {
                        // b_0 += a_0 ln t - s_0; only Re ln t = ln|t| reaches phi and E
                        // (a_0 is real for real charges, Im b_0 never enters L2P)
                        double a0_re = moment_re[src * w], a0_im = moment_im[src * w];
                        double log_re = 0.5 * log(t2);
                        b_re[j] += a0_re * log_re - s_re;
                        b_im[j] += a0_im * log_re - s_im;
                    } else {
                        double sign = (l & 1) ? 1.0 : -1.0;
                        b_re[j] += sign * (s_re * pw_re[j] - s_im * pw_im[j]);
                        b_im[j] += sign * (s_re * pw_im[j] + s_im * pw_re[j]);
                    }
                }
            }
            __syncwarp();
        }
#pragma unroll
        for (int j = 0; j < CPL; ++j) {
            for (int off = G; off < 32; off <<= 1) {
                b_re[j] += __shfl_xor_sync(0xffffffffu, b_re[j], off);
                b_im[j] += __shfl_xor_sync(0xffffffffu, b_im[j], off);
            }
            int l = li + j * G;
            if (g == 0 && l < w) {
                local_re[dst * w + l] += b_re[j];
                local_im[dst * w + l] += b_im[j];
            }
        }
    }
}

// L2L into one level, b_m(child) += sum_{l>=m} C(l, m) b_l(parent) s^(l-m), s = c_child -
// c_parent: thread per (child, m) over the level's non-empty nodes (an empty cell needs
// no local expansion), the parent from node_parent.
__global__ void k_l2l_log_level(i64 lo, i64 hi, int order, const double* __restrict__ center,
                                const int* __restrict__ parent, const i64* __restrict__ start,
                                const i64* __restrict__ end, const double* __restrict__ binomial,
                                int bsize, double* __restrict__ local_re,
                                double* __restrict__ local_im) {
    td3_chain_wait();
    td3_chain_release();
    const unsigned w = (unsigned)order + 1u;
    // (child, coefficient) from a 32-bit thread index (a level's (hi - lo) w < 2^32)
    const unsigned t = blockIdx.x * blockDim.x + threadIdx.x, tc = t / w;
    i64 ch = lo + (i64)tc;
    if (ch >= hi || end[ch] == start[ch]) return;
    int m = (int)(t - tc * w);
    i64 node = parent[ch];
    double s_re = center[2 * ch] - center[2 * node];
    double s_im = center[2 * ch + 1] - center[2 * node + 1];
    double acc_re = 0.0, acc_im = 0.0, p_re = 1.0, p_im = 0.0;
    for (int l = m; l <= order; ++l) {
        double cb = binomial[l * bsize + m];
        double b_re = local_re[node * w + l] * cb;
        double b_im = local_im[node * w + l] * cb;
        acc_re += b_re * p_re - b_im * p_im;
        acc_im += b_re * p_im + b_im * p_re;
        double nr = p_re * s_re - p_im * s_im;
        p_im = p_re * s_im + p_im * s_re;
        p_re = nr;
    }
    local_re[ch * w + m] += acc_re;
    local_im[ch * w + m] += acc_im;
}

// The downward pass in one launch: the local expansion of every non-empty leaf is its
// own M2L local plus the own M2L local of each of its ancestors shifted straight to the
// leaf's centre, b_m(leaf) += sum_{l>=m} C(l, m) b_l(a) s^(l-m), s = c_leaf - c_a.  The
// shift re-expands a polynomial exactly, so the sum equals the level-by-level L2L of the
// reference (K/fmm_downward/fmm_downward_pyccel.py:15-64) up to rounding; internal
// cells keep their own M2L locals (L2P reads leaves only).  A warp per node (non-leaves
// and empty leaves leave at once), a lane per coefficient m; the ancestors in order
// from the parent up, a fixed order per leaf.
__global__ void k_l2l_leaves(i64 count, int order, const double* __restrict__ center,
                             const int* __restrict__ parent, const i64* __restrict__ start,
                             const i64* __restrict__ end, const i64* __restrict__ child,
                             const double* __restrict__ binomial, int bsize,
                             double* __restrict__ local_re, double* __restrict__ local_im) {
    const int lane = threadIdx.x & 31;
    const int w = order + 1;
    const i64 warps = (i64)gridDim.x * (blockDim.x >> 5);
    for (i64 leaf = (i64)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); leaf < count;
         leaf += warps) {
        if (child[leaf] >= 0 || end[leaf] == start[leaf]) continue;
        const double cx = center[2 * leaf], cy = center[2 * leaf + 1];
        for (int m0 = 0; m0 < w; m0 += 32) {
            const int m = m0 + lane;
            double acc_re = 0.0, acc_im = 0.0;
            for (int a = parent[leaf]; a >= 0; a = parent[a]) {
                if (m >= w) continue;
                double s_re = cx - center[2 * a], s_im = cy - center[2 * a + 1];
                double p_re = 1.0, p_im = 0.0;
                const double* bre = local_re + (i64)a * w;
                const double* bim = local_im + (i64)a * w;
                for (int l = m; l <= order; ++l) {
                    double cb = binomial[l * bsize + m];
                    double b_re = bre[l] * cb, b_im = bim[l] * cb;
                    acc_re += b_re * p_re - b_im * p_im;
                    acc_im += b_re * p_im + b_im * p_re;
                    double nr = p_re * s_re - p_im * s_im;
                    p_im = p_re * s_im + p_im * s_re;
                    p_re = nr;
                }
            }
            if (m < w) {
                local_re[leaf * w + m] += acc_re;
                local_im[leaf * w + m] += acc_im;
            }
        }
    }
}

__global__ void k_node_parents(i64 count, const i64* __restrict__ node_child,
                               int* __restrict__ parent) {
    i64 p = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= count) return;
    if (p == 0) parent[0] = -1;
    i64 c = node_child[p];
    if (c >= 0)
        for (int k = 0; k < 4; ++k) parent[c + k] = (int)p;
}

// ------------------------------------------------------------------ mixed precision
// Moments scaled by the cell size, hat_k = a_k / h^k (|hat_k| <= sum |q|), in FP32, in
// rows of td3_hat_width(order) pairs (16-byte aligned rows; the pad pair is zero).
__global__ void k_scale_moments(i64 count, int order, const double* __restrict__ mre,
                                const double* __restrict__ mim, const double* __restrict__ half,
                                float2* __restrict__ hat) {
    td3_chain_wait();
    td3_chain_release();
    int w = order + 1, hw = td3_hat_width(order);
    i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count * hw) return;
    i64 node = t / hw;
    int k = (int)(t % hw);
    if (k >= w) {
        hat[t] = make_float2(0.0f, 0.0f);
        return;
    }
    double inv = 1.0 / half[node], s = 1.0;
    for (int j = 0; j < k; ++j) s *= inv;
    hat[t] = make_float2((float)(mre[node * w + k] * s), (float)(mim[node * w + k] * s));
}

template <int P>
struct CoefTable {
    float c[(P + 1) * (P + 1)];
};

// M2L in FP32 on the CUDA cores, one lane per translation (CSR entry), the entries of
// a warp's run of rows taken 32 at a time across row boundaries, each round's sums taken
// by columns (m2l_rows.cuh, column_round).
// With w = 1/t, ws = h_src w and wd = h_dst w (|ws|, |wd| < 1 for separated cells):
//   a'_k = hat_k ws^k,  s_l = sum_k coeff[k, l] a'_k,
//   bhat_0 = a_0 ln|t| - s_0,  bhat_l = -(-1)^l s_l wd^l  (b_l = bhat_l / h_dst^l),
// the reference's translation with every quantity O(1).  ln|t| is taken in units of
// `unit` (L): a_0 ln|t| = a_0 ln|t / L| + a_0 ln L, the second summed over the partners
// and added in FP64.  The coefficient matrix is a kernel parameter (constant bank).
template <int P>
__global__ void __launch_bounds__(32 * M2L_WARPS)
k_m2l_mixed(const i64* __restrict__ row_start, const int* __restrict__ entry_row,
            const i64* __restrict__ partners, i64 n_dst, const double* __restrict__ dst_center,
            const double* __restrict__ dst_half, const double* __restrict__ src_center,
            const double* __restrict__ src_half, const float2* __restrict__ hat, int order,
            const CoefTable<P> C, double unit, double* __restrict__ local_re,
            double* __restrict__ local_im) {
    td3_chain_wait();
    td3_chain_release();
    constexpr int W = P + 1, V = 2 * W + 2;
    __shared__ __align__(16) float stage[M2L_WARPS][32 * V];
    int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    int w = order + 1;
    double inv_unit2 = 1.0 / (unit * unit), ln_unit = log(unit);
    i64 e0, e1;
    td3m2l::warp_entries(row_start, n_dst, (i64)blockIdx.x * M2L_WARPS + wib,
                         (i64)gridDim.x * M2L_WARPS, e0, e1);
    float col[(V + 31) / 32], comp[(V + 31) / 32];
#pragma unroll
    for (int c = 0; c < (V + 31) / 32; ++c) col[c] = comp[c] = 0.0f;
    for (i64 base = e0; base < e1; base += 32) {
        i64 e = base + lane;
        bool live = e < e1;
        int d = live ? entry_row[e] : -1;
        float v[V];
#pragma unroll
        for (int j = 0; j < V; ++j) v[j] = 0.0f;
        if (live) {
            i64 src = partners[e];
            double cx = dst_center[2 * d], cy = dst_center[2 * d + 1], hd = dst_half[d];
            double tr = cx - src_center[2 * src], ti = cy - src_center[2 * src + 1];
            double t2 = tr * tr + ti * ti, inv = 1.0 / t2, hs = src_half[src];
            float wsr = (float)(hs * tr * inv), wsi = (float)(-hs * ti * inv);
            float wdr = (float)(hd * tr * inv), wdi = (float)(-hd * ti * inv);
            float lnt = 0.5f * log_split(t2 * inv_unit2);
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
            float ar[W], ai[W];
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
            float qr = 1.0f, qi = 0.0f;
#pragma unroll
            for (int l = 0; l < W; ++l) {
                float sr = 0.0f, si = 0.0f;
#pragma unroll
                for (int k = 0; k < W; ++k) {
                    sr += C.c[k * W + l] * ar[k];
                    si += C.c[k * W + l] * ai[k];
                }
                if (l == 0) {
                    v[0] = ar[0] * lnt - sr;
                    v[1] = ai[0] * lnt - si;
                } else {
                    float sign = (l & 1) ? 1.0f : -1.0f;
                    v[2 * l] = sign * (sr * qr - si * qi);
                    v[2 * l + 1] = sign * (sr * qi + si * qr);
                }
                float nr = qr * wdr - qi * wdi;
                qi = qr * wdi + qi * wdr;
                qr = nr;
            }
            v[2 * W] = ar[0];
            v[2 * W + 1] = ai[0];
        }
        td3m2l::column_round<W>(v, d, live, lane, base + 32, e1, entry_row, w, dst_half, ln_unit,
                                local_re, local_im, stage[wib], col, comp);
    }
}

template <int P>
int launch_m2l_mixed(const i64* row_start, const int* entry_row, const i64* partners, i64 n_dst,
                     const double* dst_center, const double* dst_half, const double* src_center,
                     const double* src_half, const float2* hat, int order, const double* coeff,
                     double unit, double* lre, double* lim, cudaStream_t s) {
    // the reference's matrix, zero-padded from (order + 1)^2 to (P + 1)^2
    CoefTable<P> C;
    int w = order + 1;
    for (int k = 0; k <= P; ++k)
        for (int l = 0; l <= P; ++l)
            C.c[k * (P + 1) + l] = (k < w && l < w) ? (float)coeff[k * w + l] : 0.0f;
    TD3_TRY(td3_launch_chained(k_m2l_mixed<P>, 148 * 16, 32 * M2L_WARPS, 0, s, row_start,
                               entry_row, partners, n_dst, dst_center, dst_half, src_center,
                               src_half, hat, order, C, unit, lre, lim));
    TD3_CHECK_LAUNCH();
    return TD3_OK;
}

template <int G, int CPL>
void launch_m2l(const i64* row_start, const i64* partners, i64 n_dst, const double* dst_center,
                const double* src_center, const double* mre, const double* mim, int order,
                const double* coeff, double* lre, double* lim, cudaStream_t s) {
    i64 blocks = (n_dst + M2L_WARPS - 1) / M2L_WARPS;
    if (blocks > 148 * 64) blocks = 148 * 64;
    k_m2l_log<G, CPL><<<(unsigned)blocks, 32 * M2L_WARPS, 0, s>>>(
        row_start, partners, n_dst, dst_center, src_center, mre, mim, order, coeff, lre, lim);
}

}  // namespace

extern "C" int td3_fmm_m2l(const int64_t* row_start, const int64_t* partners, int64_t n_dst,
                           const double* dst_center, const double* src_center,
                           const double* moment_re, const double* moment_im, int order,
                           const double* coeff, double* local_re, double* local_im, void* stream) {
    if (n_dst < 0 || order < 0 || order > TD3_MAX_ORDER) return TD3_EINVAL;
    if (n_dst == 0) return TD3_OK;
    cudaStream_t s = td3_stream(stream);
    int w = order + 1;
    if (w <= 8)
        launch_m2l<8, 1>(row_start, partners, n_dst, dst_center, src_center, moment_re, moment_im,
                         order, coeff, local_re, local_im, s);
    else if (w <= 16)
        launch_m2l<16, 1>(row_start, partners, n_dst, dst_center, src_center, moment_re, moment_im,
                          order, coeff, local_re, local_im, s);
    else if (w <= 32)
        launch_m2l<32, 1>(row_start, partners, n_dst, dst_center, src_center, moment_re, moment_im,
                          order, coeff, local_re, local_im, s);
    else
        launch_m2l<32, 3>(row_start, partners, n_dst, dst_center, src_center, moment_re, moment_im,
                          order, coeff, local_re, local_im, s);
    TD3_CHECK_LAUNCH();
    return TD3_OK;
}

extern "C" int td3_scale_moments(int64_t count, int order, const double* moment_re,
                                 const double* moment_im, const double* node_half, float* hat,
                                 void* stream) {
    if (count < 0 || order < 0 || order > TD3_MAX_ORDER) return TD3_EINVAL;
    if (count == 0) return TD3_OK;
    i64 threads = count * td3_hat_width(order);
    TD3_TRY(td3_launch_chained(k_scale_moments, td3_blocks(threads, 256), 256, 0,
                               td3_stream(stream), count, order, moment_re, moment_im, node_half,
                               reinterpret_cast<float2*>(hat)));
    TD3_CHECK_LAUNCH();
    return TD3_OK;
}

extern "C" int td3_fmm_m2l_mixed(const int64_t* row_start, const int32_t* entry_row,
                                 const int64_t* partners, int64_t n_dst,
                                 const double* dst_center, const double* dst_half,
                                 const double* src_center, const double* src_half,
                                 const float* hat, int order, const double* coeff, double unit,
                                 int tensor_cores, double* local_re, double* local_im,
                                 int64_t* status, void* stream) {
    if (n_dst < 0 || order < 0 || order > 20) return TD3_EINVAL;
    if (!(unit > 0.0 && unit < INFINITY)) return TD3_EINVAL;
    if (tensor_cores && !status) return TD3_EINVAL;
    if (n_dst == 0) return TD3_OK;
    cudaStream_t s = td3_stream(stream);
    const float2* h = reinterpret_cast<const float2*>(hat);
    if (tensor_cores && order <= 15)
        return td3_m2l_tensor(row_start, entry_row, partners, n_dst, dst_center, dst_half, src_center,
                              src_half, h, order, coeff, unit, local_re, local_im, status, s);
    if (order <= 4)
        return launch_m2l_mixed<4>(row_start, entry_row, partners, n_dst, dst_center, dst_half, src_center,
                                   src_half, h, order, coeff, unit, local_re, local_im, s);
    if (order <= 8)
        return launch_m2l_mixed<8>(row_start, entry_row, partners, n_dst, dst_center, dst_half, src_center,
                                   src_half, h, order, coeff, unit, local_re, local_im, s);
    if (order <= 12)
        return launch_m2l_mixed<12>(row_start, entry_row, partners, n_dst, dst_center, dst_half, src_center,
                                    src_half, h, order, coeff, unit, local_re, local_im, s);
    if (order <= 16)
        return launch_m2l_mixed<16>(row_start, entry_row, partners, n_dst, dst_center, dst_half, src_center,
                                    src_half, h, order, coeff, unit, local_re, local_im, s);
    return launch_m2l_mixed<20>(row_start, entry_row, partners, n_dst, dst_center, dst_half, src_center,
                                src_half, h, order, coeff, unit, local_re, local_im, s);
}

extern "C" int td3_node_parents(int64_t count, const int64_t* node_child, int32_t* node_parent,
                                void* stream) {
    if (count < 1 || count > 0x7fffffffLL) return TD3_EINVAL;
    k_node_parents<<<td3_blocks(count, 256), 256, 0, td3_stream(stream)>>>(count, node_child,
                                                                          node_parent);
    TD3_CHECK_LAUNCH();
    return TD3_OK;
}

extern "C" int td3_fmm_downward(const int64_t* levels, int64_t n_levels, const double* node_center,
                                const int32_t* node_parent, const int64_t* node_start,
                                const int64_t* node_end, int order, const double* binomial,
                                int binomial_size, double* local_re, double* local_im,
                                void* stream) {
    if (n_levels < 1 || order < 0 || order > TD3_MAX_ORDER || binomial_size < order + 1)
        return TD3_EINVAL;
    cudaStream_t s = td3_stream(stream);
    int w = order + 1;
    for (i64 level = 1; level < n_levels; ++level) {
        i64 lo = levels[level], hi = levels[level + 1];
        if (hi <= lo) continue;
        i64 threads = (hi - lo) * w;
        if (threads > 0xffffffffLL) return TD3_EINVAL;
        TD3_TRY(td3_launch_chained(k_l2l_log_level, td3_blocks(threads, 256), 256, 0, s, lo, hi,
                                   order, node_center, node_parent, node_start, node_end,
                                   binomial, binomial_size, local_re, local_im));
    }
    TD3_CHECK_LAUNCH();
    return TD3_OK;
}

extern "C" int td3_fmm_downward_leaves(int64_t count, int order, const double* node_center,
                                       const int32_t* node_parent, const int64_t* node_start,
                                       const int64_t* node_end, const int64_t* node_child,
                                       const double* binomial, int binomial_size,
                                       double* local_re, double* local_im, void* stream) {
    if (count < 1 || count > 0x7fffffffLL || order < 0 || order > TD3_MAX_ORDER ||
        binomial_size < order + 1)
        return TD3_EINVAL;
    constexpr int threads = 256;
    i64 blocks = (count + threads / 32 - 1) / (threads / 32);
    if (blocks > 148 * 32) blocks = 148 * 32;
    k_l2l_leaves<<<(unsigned)blocks, threads, 0, td3_stream(stream)>>>(
        count, order, node_center, node_parent, node_start, node_end, node_child, binomial,
        binomial_size, local_re, local_im);
    TD3_CHECK_LAUNCH();
    return TD3_OK;
}
