// The FMM of the line-charge (log) kernel in complex form (Greengard-Rokhlin), FP64:
//   M2L by destination row    (K/fmm_m2l_host/fmm_m2l_host_pyccel.py:16-105; GPU form
//                              K/fmm_m2l/fmm_m2l_cuda.cu:12-80)
//   L2L per level             (K/fmm_downward/fmm_downward_pyccel.py:15-64)
//   L2P + near field P2P      (K/fmm_evaluate_host/fmm_evaluate_host_pyccel.py:14-100;
//                              K/fmm_evaluate/fmm_evaluate_cuda.cu:11-87)
//   targets of fmm_at         (K/log_targets_host/log_targets_host_pyccel.py:14-94)
//
// M2L: one warp per destination cell; the warp splits into groups of G lanes, lane l
// of a group owning expansion coefficient l (and l + G), each group taking every
// (32/G)-th partner; the scaled moments a'_k = a_k w^k pass through shared memory and
// s_l = sum_k coeff[k, l] a'_k is the real matrix product of the reference.  The
// partial locals of the groups are summed by shuffles and added once per cell.
// P2P: one warp per target leaf, lanes split into (target, source slice); each target
// sums its own row of partners, so the near field needs no atomics and no mutual
// writes (each pair is evaluated from both sides).
#include "common.cuh"

namespace {

constexpr int M2L_WARPS = 4;
constexpr int EVAL_WARPS = 4;

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

// L2L of one level: thread per (node, child, m).
__global__ void k_l2l_log(i64 lo, i64 hi, int order, const double* __restrict__ center,
                          const i64* __restrict__ child, const double* __restrict__ binomial,
                          int bsize, double* __restrict__ local_re, double* __restrict__ local_im) {
    int w = order + 1;
    i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    i64 node = lo + t / (4 * w);
    if (node >= hi) return;
    i64 first = child[node];
    if (first < 0) return;
    int c = (int)((t / w) % 4), m = (int)(t % w);
    i64 ch = first + c;
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

// Horner evaluation of the local expansion at u: W and W' (fmm_evaluate_host_pyccel.py:48-60).
__device__ __forceinline__ void l2p_log(const double* __restrict__ lre, const double* __restrict__ lim,
                                        int order, double u_re, double u_im, double& w_re,
                                        double& w_im, double& d_re, double& d_im) {
    w_re = lre[order];
    w_im = lim[order];
    d_re = 0.0;
    d_im = 0.0;
    for (int l = order - 1; l >= 0; --l) {
        double nd_re = d_re * u_re - d_im * u_im + w_re;
        d_im = d_re * u_im + d_im * u_re + w_im;
        d_re = nd_re;
        double nw_re = w_re * u_re - w_im * u_im + lre[l];
        w_im = w_re * u_im + w_im * u_re + lim[l];
        w_re = nw_re;
    }
}

__device__ __forceinline__ int pow2_at_least(int v) {
    int p = 1;
    while (p < v) p <<= 1;
    return p;
}

// L2P + P2P at the particles of every leaf (targets = sources, in tree order); the
// results are written at the particles' input indices perm[k].
template <bool POT>
__global__ void __launch_bounds__(32 * EVAL_WARPS)
k_eval_log(const double* __restrict__ spos, const double* __restrict__ scharge,
           const i64* __restrict__ perm, i64 n, i64 node_count, const double* __restrict__ center,
           const i64* __restrict__ start, const i64* __restrict__ end, const i64* __restrict__ child,
           int order, const double* __restrict__ local_re, const double* __restrict__ local_im,
           const i64* __restrict__ p2p_rows, const i64* __restrict__ p2p_partners, double eps2,
           double* __restrict__ phi, double* __restrict__ field, i64* status) {
    int lane = threadIdx.x & 31;
    i64 leaf = (i64)blockIdx.x * EVAL_WARPS + (threadIdx.x >> 5);
    if (leaf >= node_count || child[leaf] >= 0) return;
    i64 s0 = start[leaf], s1 = end[leaf];
    int count = (int)(s1 - s0);
    if (count <= 0) return;
    int tsz = pow2_at_least(count < 32 ? count : 32);
    int slices = 32 / tsz;
    int ti = lane % tsz, slice = lane / tsz;
    int w = order + 1;
    double cx = center[2 * leaf], cy = center[2 * leaf + 1];
    i64 r0 = p2p_rows[leaf], r1 = p2p_rows[leaf + 1];
    for (int base = 0; base < count; base += tsz) {
        int it = base + ti;
        bool valid = it < count;
        i64 k = s0 + (valid ? it : 0);
        double xi = spos[k], yi = spos[n + k], qi = scharge[k];
        double pot = 0.0, ex = 0.0, ey = 0.0;
        bool bad = false;
        if (valid) {
            for (i64 e = r0; e < r1; ++e) {
                i64 b = p2p_partners[e];
                i64 b0 = start[b], b1 = end[b];
                for (i64 j = b0 + slice; j < b1; j += slices) {
                    if (j == k) continue;
                    double qj = scharge[j];
                    double dx = xi - spos[j], dy = yi - spos[n + j];
                    double r2 = dx * dx + dy * dy + eps2;
                    if (r2 == 0.0) {
                        bad |= (qi != 0.0 && qj != 0.0);
                        continue;
                    }
                    if (POT) pot -= qj * log(r2);
                    double f = 2.0 * qj / r2;
                    ex += f * dx;
                    ey += f * dy;
                }
            }
        }
        for (int off = tsz; off < 32; off <<= 1) {
            pot += __shfl_xor_sync(0xffffffffu, pot, off);
            ex += __shfl_xor_sync(0xffffffffu, ex, off);
            ey += __shfl_xor_sync(0xffffffffu, ey, off);
        }
        if (valid && slice == 0) {
            double w_re, w_im, d_re, d_im;
            l2p_log(local_re + leaf * w, local_im + leaf * w, order, xi - cx, yi - cy, w_re, w_im,
                    d_re, d_im);
            i64 i = perm[k];
            phi[i] = POT ? (-2.0 * w_re + pot) : 0.0;
            field[i] = 2.0 * d_re + ex;
            field[n + i] = -2.0 * d_im + ey;
        }
        // any slice that met a coincident charged pair reports the target
        unsigned badmask = __ballot_sync(0xffffffffu, bad && valid);
        if (badmask && lane == __ffs(badmask) - 1) td3_report(status, perm[k] + 1);
    }
}

// fmm_at, log kernel: L2P at the target leaves plus exact sums over the partner source
// leaves, skipping source exclude (an index of the source perm); phi 1e300 marks a
// coincident charge (log_targets_host_pyccel.py:14-94).  Results at input indices.
template <bool POT>
__global__ void __launch_bounds__(32 * EVAL_WARPS)
k_targets_log(const double* __restrict__ tpos, const i64* __restrict__ texclude,
              const i64* __restrict__ tperm, i64 m, i64 t_count, const double* __restrict__ t_center,
              const i64* __restrict__ t_start, const i64* __restrict__ t_end,
              const i64* __restrict__ t_child, int order, const double* __restrict__ local_re,
              const double* __restrict__ local_im, const i64* __restrict__ rows,
              const i64* __restrict__ partners, const double* __restrict__ spos,
              const double* __restrict__ scharge, const i64* __restrict__ sindex, i64 n,
              const i64* __restrict__ s_start, const i64* __restrict__ s_end, double eps2,
              double* __restrict__ phi, double* __restrict__ field, i64* status) {
    int lane = threadIdx.x & 31;
    i64 leaf = (i64)blockIdx.x * EVAL_WARPS + (threadIdx.x >> 5);
    if (leaf >= t_count || t_child[leaf] >= 0) return;
    i64 s0 = t_start[leaf], s1 = t_end[leaf];
    int count = (int)(s1 - s0);
    if (count <= 0) return;
    int tsz = pow2_at_least(count < 32 ? count : 32);
    int slices = 32 / tsz;
    int ti = lane % tsz, slice = lane / tsz;
    int w = order + 1;
    double cx = t_center[2 * leaf], cy = t_center[2 * leaf + 1];
    i64 r0 = rows[leaf], r1 = rows[leaf + 1];
    for (int base = 0; base < count; base += tsz) {
        int it = base + ti;
        bool valid = it < count;
        i64 k = s0 + (valid ? it : 0);
        double xi = tpos[k], yi = tpos[m + k];
        i64 skip = texclude[k];
        double pot = 0.0, ex = 0.0, ey = 0.0;
        bool bad = false;
        if (valid) {
            for (i64 e = r0; e < r1; ++e) {
                i64 b = partners[e];
                for (i64 j = s_start[b] + slice; j < s_end[b]; j += slices) {
                    double c = scharge[j];
                    if (c == 0.0 || sindex[j] == skip) continue;
                    double dx = xi - spos[j], dy = yi - spos[n + j];
                    double r2 = dx * dx + dy * dy + eps2;
                    if (r2 == 0.0) {
                        bad = true;
                        continue;
                    }
                    if (POT) pot -= c * log(r2);
                    double f = 2.0 * c / r2;
                    ex += f * dx;
                    ey += f * dy;
                }
            }
        }
        for (int off = tsz; off < 32; off <<= 1) {
            pot += __shfl_xor_sync(0xffffffffu, pot, off);
            ex += __shfl_xor_sync(0xffffffffu, ex, off);
            ey += __shfl_xor_sync(0xffffffffu, ey, off);
        }
        unsigned badmask = __ballot_sync(0xffffffffu, bad && valid);
        i64 i = tperm[k];
        if (valid && slice == 0) {
            double w_re, w_im, d_re, d_im;
            l2p_log(local_re + leaf * w, local_im + leaf * w, order, xi - cx, yi - cy, w_re, w_im,
                    d_re, d_im);
            phi[i] = POT ? (-2.0 * w_re + pot) : 0.0;
            field[i] = 2.0 * d_re + ex;
            field[m + i] = -2.0 * d_im + ey;
        }
        if (badmask && lane == __ffs(badmask) - 1) td3_report(status, i + 1);
    }
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

extern "C" int td3_fmm_downward(const int64_t* levels, int64_t n_levels, const double* node_center,
                                const int64_t* node_child, int order, const double* binomial,
                                int binomial_size, double* local_re, double* local_im,
                                void* stream) {
    if (n_levels < 1 || order < 0 || order > TD3_MAX_ORDER || binomial_size < order + 1)
        return TD3_EINVAL;
    cudaStream_t s = td3_stream(stream);
    int w = order + 1;
    for (i64 level = 0; level + 1 < n_levels; ++level) {
        i64 lo = levels[level], hi = levels[level + 1];
        if (hi <= lo) continue;
        i64 threads = (hi - lo) * 4 * w;
        k_l2l_log<<<td3_blocks(threads, 256), 256, 0, s>>>(lo, hi, order, node_center, node_child,
                                                            binomial, binomial_size, local_re,
                                                            local_im);
    }
    TD3_CHECK_LAUNCH();
    return TD3_OK;
}

extern "C" int td3_fmm_evaluate(const double* sorted_pos, const double* sorted_charge,
                                const int64_t* perm, int64_t n, int64_t node_count,
                                const double* node_center, const int64_t* node_start,
                                const int64_t* node_end, const int64_t* node_child, int order,
                                const double* local_re, const double* local_im,
                                const int64_t* p2p_rows, const int64_t* p2p_partners,
                                double softening, int with_potential, double* phi, double* field,
                                int64_t* status, void* stream) {
    if (n < 0 || node_count < 1 || order < 0 || order > TD3_MAX_ORDER) return TD3_EINVAL;
    if (n == 0) return TD3_OK;
    cudaStream_t s = td3_stream(stream);
    unsigned blocks = td3_blocks(node_count, EVAL_WARPS);
    double eps2 = softening * softening;
    if (with_potential)
        k_eval_log<true><<<blocks, 32 * EVAL_WARPS, 0, s>>>(
            sorted_pos, sorted_charge, perm, n, node_count, node_center, node_start, node_end,
            node_child, order, local_re, local_im, p2p_rows, p2p_partners, eps2, phi, field, status);
    else
        k_eval_log<false><<<blocks, 32 * EVAL_WARPS, 0, s>>>(
            sorted_pos, sorted_charge, perm, n, node_count, node_center, node_start, node_end,
            node_child, order, local_re, local_im, p2p_rows, p2p_partners, eps2, phi, field, status);
    TD3_CHECK_LAUNCH();
    return TD3_OK;
}

extern "C" int td3_log_targets(const double* sorted_targets, const int64_t* sorted_exclude,
                               const int64_t* target_perm, int64_t m, int64_t t_count,
                               const double* t_center, const int64_t* t_start,
                               const int64_t* t_end, const int64_t* t_child, int order,
                               const double* local_re, const double* local_im,
                               const int64_t* rows, const int64_t* partners,
                               const double* sorted_pos, const double* sorted_charge,
                               const int64_t* perm, int64_t n, const int64_t* s_start,
                               const int64_t* s_end, double softening, int with_potential,
                               double* phi, double* field, int64_t* status, void* stream) {
    if (m < 0 || n < 0 || t_count < 1 || order < 0 || order > TD3_MAX_ORDER) return TD3_EINVAL;
    if (m == 0) return TD3_OK;
    cudaStream_t s = td3_stream(stream);
    unsigned blocks = td3_blocks(t_count, EVAL_WARPS);
    double eps2 = softening * softening;
    if (with_potential)
        k_targets_log<true><<<blocks, 32 * EVAL_WARPS, 0, s>>>(
            sorted_targets, sorted_exclude, target_perm, m, t_count, t_center, t_start, t_end,
            t_child, order, local_re, local_im, rows, partners, sorted_pos, sorted_charge, perm, n,
            s_start, s_end, eps2, phi, field, status);
    else
        k_targets_log<false><<<blocks, 32 * EVAL_WARPS, 0, s>>>(
            sorted_targets, sorted_exclude, target_perm, m, t_count, t_center, t_start, t_end,
            t_child, order, local_re, local_im, rows, partners, sorted_pos, sorted_charge, perm, n,
            s_start, s_end, eps2, phi, field, status);
    TD3_CHECK_LAUNCH();
    return TD3_OK;
}
