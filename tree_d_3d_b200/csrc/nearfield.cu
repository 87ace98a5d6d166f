// Near field of the FMM (P2P) fused with the evaluation of the local expansions (L2P):
//   at the sources, log kernel   K/fmm_evaluate_host/fmm_evaluate_host_pyccel.py:14-100
//   at the sources, Coulomb      K/cart_evaluate_host/cart_evaluate_host_pyccel.py:16-110
//   at other targets (fmm_at)    K/log_targets_host/log_targets_host_pyccel.py:14-94,
//                                K/cart_targets_host/cart_targets_host_pyccel.py:16-98
//
// Target-centric: every target sums its own leaf's partner leaves, so each pair is
// evaluated from both sides and nothing is written by two threads.  Partner rows are
// very uneven (a coarse leaf beside a dense cluster has thousands of partners), so
// td3_nearfield_plan cuts each leaf's row into segments of at most `segment`
// partners; one warp takes one segment (lanes = targets x partner slices).  A leaf
// with one segment writes its final values; the segments of a longer row write
// partial sums that a finish pass adds in segment order (deterministic results).
#include "common.cuh"

namespace {

constexpr int NF_WARPS = 4;
constexpr int LOCAL_COMPLEX = 0;
constexpr int LOCAL_CART = 1;

__device__ __forceinline__ int pow2_at_least(int v) {
    int p = 1;
    while (p < v) p <<= 1;
    return p;
}

// ------------------------------------------------------------------ the plan
__global__ void k_plan_count(i64 n_nodes, const i64* __restrict__ rows, const i64* __restrict__ child,
                             const i64* __restrict__ start, const i64* __restrict__ end, int segment,
                             i64* __restrict__ nseg, i64* __restrict__ psize) {
    i64 n = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= n_nodes) return;
    i64 count = end[n] - start[n];
    i64 s = 0;
    if (child[n] < 0 && count > 0) {
        i64 len = rows[n + 1] - rows[n];
        s = len <= segment ? 1 : (len + segment - 1) / segment;
    }
    nseg[n] = s;
    psize[n] = s > 1 ? s * count : 0;
}

__global__ void k_plan_fill(i64 n_nodes, const i64* __restrict__ rows, const i64* __restrict__ start,
                            const i64* __restrict__ end, int segment,
                            const i64* __restrict__ nseg_scan, const i64* __restrict__ psize_scan,
                            const i64* __restrict__ nseg, int* __restrict__ seg_leaf,
                            longlong2* __restrict__ seg_range, i64* __restrict__ seg_out) {
    i64 n = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= n_nodes) return;
    i64 s = nseg[n];
    if (s == 0) return;
    i64 first = nseg_scan[n], count = end[n] - start[n];
    i64 r0 = rows[n], r1 = rows[n + 1];
    for (i64 k = 0; k < s; ++k) {
        i64 e0 = r0 + k * segment;
        i64 e1 = e0 + segment < r1 ? e0 + segment : r1;
        if (s == 1) e1 = r1;
        seg_leaf[first + k] = (int)n;
        seg_range[first + k] = make_longlong2(e0, e1);
        seg_out[first + k] = s > 1 ? psize_scan[n] + k * count : -1;
    }
}

// ------------------------------------------------------------------ local expansions
// Log kernel: W and W' of the complex local expansion at u (Horner, the reference order).
__device__ __forceinline__ void l2p_complex(const double* __restrict__ lre,
                                            const double* __restrict__ lim, int order, double ux,
                                            double uy, double& phi, double& fx, double& fy) {
    double w_re = lre[order], w_im = lim[order], d_re = 0.0, d_im = 0.0;
    for (int l = order - 1; l >= 0; --l) {
        double nd_re = d_re * ux - d_im * uy + w_re;
        d_im = d_re * uy + d_im * ux + w_im;
        d_re = nd_re;
        double nw_re = w_re * ux - w_im * uy + lre[l];
        w_im = w_re * uy + w_im * ux + lim[l];
        w_re = nw_re;
    }
    phi = -2.0 * w_re;
    fx = 2.0 * d_re;
    fy = -2.0 * d_im;
}

// Coulomb: phi(c + u) = sum_b uy^b P_b(ux), P_b(x) = sum_a T[(a, b)] x^a, evaluated by
// nested Horner together with both derivatives; E = -grad phi.
__device__ __forceinline__ void l2p_cart(const double* __restrict__ T, int order, double ux,
                                         double uy, double& phi, double& fx, double& fy) {
    double q = 0.0, dq = 0.0, g = 0.0;
    for (int b = order; b >= 0; --b) {
        int top = order - b;  // highest power of x in P_b
        // coefficient (a, b) sits at n (n + 1) / 2 + b with n = a + b
        int n = top + b;
        double p = T[n * (n + 1) / 2 + b], dp = 0.0;
        for (int a = top - 1; a >= 0; --a) {
            n = a + b;
            dp = dp * ux + p;
            p = p * ux + T[n * (n + 1) / 2 + b];
        }
        dq = dq * uy + q;
        q = q * uy + p;
        g = g * uy + dp;
    }
    phi = q;
    fx = -g;
    fy = -dq;
}

template <int LOCAL>
__device__ __forceinline__ void eval_local(const double* __restrict__ local_a,
                                           const double* __restrict__ local_b, i64 leaf, int order,
                                           int width, double ux, double uy, double& phi,
                                           double& fx, double& fy) {
    if (LOCAL == LOCAL_COMPLEX)
        l2p_complex(local_a + leaf * width, local_b + leaf * width, order, ux, uy, phi, fx, fy);
    else
        l2p_cart(local_a + leaf * width, order, ux, uy, phi, fx, fy);
}

struct Sources {
    const double* pos;     // (2, n) tree order
    const double* charge;  // (n) tree order
    const i64* index;      // (n) input index of each slot (exclusion)
    const i64* start;
    const i64* end;
    i64 n;
};

struct Targets {
    const double* pos;     // (2, m) tree order
    const i64* exclude;    // (m) tree order, may be null (at the sources: the slot itself)
    const i64* perm;       // (m) input index of each slot
    const double* center;  // target tree cells
    const i64* start;
    const i64* end;
    i64 m;
};

// One warp per segment.  OTHER: targets and sources are different point sets (fmm_at):
// zero charges and source exclude[i] are skipped and any coincidence is an error.
// Otherwise targets are the sources themselves: a particle skips itself and a
// coincident pair is an error only if both charges are nonzero.
template <int KERNEL, bool POT, bool OTHER, int LOCAL>
__global__ void __launch_bounds__(32 * NF_WARPS)
k_near(Targets T, Sources S, i64 n_seg, const int* __restrict__ seg_leaf,
       const longlong2* __restrict__ seg_range, const i64* __restrict__ seg_out,
       const i64* __restrict__ partners, const double* __restrict__ local_a,
       const double* __restrict__ local_b, int order, int width, double eps2,
       double* __restrict__ partial, double* __restrict__ phi, double* __restrict__ field,
       i64* status) {
    int lane = threadIdx.x & 31;
    i64 seg = (i64)blockIdx.x * NF_WARPS + (threadIdx.x >> 5);
    if (seg >= n_seg) return;
    i64 leaf = seg_leaf[seg];
    longlong2 er = seg_range[seg];
    i64 outp = seg_out[seg];
    i64 s0 = T.start[leaf];
    int count = (int)(T.end[leaf] - s0);
    int tsz = pow2_at_least(count < 32 ? count : 32);
    int slices = 32 / tsz;
    int ti = lane % tsz, slice = lane / tsz;
    for (int base = 0; base < count; base += tsz) {
        int it = base + ti;
        bool valid = it < count;
        i64 k = s0 + (valid ? it : 0);
        double xi = T.pos[k], yi = T.pos[T.m + k];
        double qi = OTHER ? 0.0 : S.charge[k];
        i64 skip = OTHER ? (T.exclude ? T.exclude[k] : -1) : k;
        double pot = 0.0, ex = 0.0, ey = 0.0;
        bool bad = false;
        if (valid) {
            for (i64 e = er.x + slice; e < er.y; e += slices) {
                i64 b = partners[e];
                i64 b1 = S.end[b];
                for (i64 j = S.start[b]; j < b1; ++j) {
                    double qj = S.charge[j];
                    if (OTHER) {
                        if (qj == 0.0 || S.index[j] == skip) continue;
                    } else if (j == skip) {
                        continue;
                    }
                    double dx = xi - S.pos[j], dy = yi - S.pos[S.n + j];
                    double r2 = dx * dx + dy * dy + eps2;
                    if (r2 == 0.0) {
                        bad |= OTHER ? true : (qi != 0.0 && qj != 0.0);
                        continue;
                    }
                    if (KERNEL == TD3_KERNEL_LOG) {
                        if (POT) pot -= qj * log(r2);
                        double f = 2.0 * qj / r2;
                        ex += f * dx;
                        ey += f * dy;
                    } else {
                        double inv_r = rsqrt(r2);
                        double inv_r3 = inv_r * inv_r * inv_r;
                        pot += qj * inv_r;
                        ex += qj * inv_r3 * dx;
                        ey += qj * inv_r3 * dy;
                    }
                }
            }
        }
        for (int off = tsz; off < 32; off <<= 1) {
            pot += __shfl_xor_sync(0xffffffffu, pot, off);
            ex += __shfl_xor_sync(0xffffffffu, ex, off);
            ey += __shfl_xor_sync(0xffffffffu, ey, off);
        }
        unsigned badmask = __ballot_sync(0xffffffffu, bad && valid);
        if (valid && slice == 0) {
            if (outp < 0) {
                double lp, lx, ly;
                eval_local<LOCAL>(local_a, local_b, leaf, order, width, xi - T.center[2 * leaf],
                                  yi - T.center[2 * leaf + 1], lp, lx, ly);
                i64 i = T.perm[k];
                phi[i] = POT ? lp + pot : 0.0;
                field[i] = lx + ex;
                field[T.m + i] = ly + ey;
            } else {
                i64 p = outp + it;
                partial[3 * p] = pot;
                partial[3 * p + 1] = ex;
                partial[3 * p + 2] = ey;
            }
        }
        if (badmask && lane == __ffs(badmask) - 1) td3_report(status, T.perm[k] + 1);
    }
}

// Leaves whose row took several segments: partial sums in segment order, plus L2P.
template <bool POT, int LOCAL>
__global__ void k_near_finish(Targets T, i64 n_seg, const int* __restrict__ seg_leaf,
                              const i64* __restrict__ seg_out, const double* __restrict__ local_a,
                              const double* __restrict__ local_b, int order, int width,
                              const double* __restrict__ partial, double* __restrict__ phi,
                              double* __restrict__ field) {
    i64 seg = (i64)blockIdx.x * NF_WARPS + (threadIdx.x >> 5);
    int lane = threadIdx.x & 31;
    if (seg >= n_seg) return;
    i64 p0 = seg_out[seg];
    // the first segment of a multi-segment leaf finishes it
    if (p0 < 0 || (seg > 0 && seg_leaf[seg - 1] == seg_leaf[seg])) return;
    i64 leaf = seg_leaf[seg];
    i64 s0 = T.start[leaf];
    int count = (int)(T.end[leaf] - s0);
    i64 last = seg;
    while (last + 1 < n_seg && seg_leaf[last + 1] == leaf) ++last;
    for (int it = lane; it < count; it += 32) {
        double pot = 0.0, ex = 0.0, ey = 0.0;
        for (i64 s = seg; s <= last; ++s) {
            i64 p = seg_out[s] + it;
            pot += partial[3 * p];
            ex += partial[3 * p + 1];
            ey += partial[3 * p + 2];
        }
        i64 k = s0 + it;
        double xi = T.pos[k], yi = T.pos[T.m + k];
        double lp, lx, ly;
        eval_local<LOCAL>(local_a, local_b, leaf, order, width, xi - T.center[2 * leaf],
                          yi - T.center[2 * leaf + 1], lp, lx, ly);
        i64 i = T.perm[k];
        phi[i] = POT ? lp + pot : 0.0;
        field[i] = lx + ex;
        field[T.m + i] = ly + ey;
    }
}

template <int KERNEL, bool POT, bool OTHER, int LOCAL>
int launch_near(const Targets& T, const Sources& S, i64 n_seg, const int* seg_leaf,
                const longlong2* seg_range, const i64* seg_out, const i64* partners,
                const double* la, const double* lb, int order, int width, double eps2,
                double* partial, double* phi, double* field, i64* status, cudaStream_t s) {
    if (n_seg == 0) return TD3_OK;
    unsigned blocks = td3_blocks(n_seg, NF_WARPS);
    k_near<KERNEL, POT, OTHER, LOCAL><<<blocks, 32 * NF_WARPS, 0, s>>>(
        T, S, n_seg, seg_leaf, seg_range, seg_out, partners, la, lb, order, width, eps2, partial,
        phi, field, status);
    k_near_finish<POT, LOCAL><<<blocks, 32 * NF_WARPS, 0, s>>>(T, n_seg, seg_leaf, seg_out, la, lb,
                                                               order, width, partial, phi, field);
    TD3_CHECK_LAUNCH();
    return TD3_OK;
}

template <bool OTHER, int LOCAL>
int dispatch_near(int kernel, int with_potential, const Targets& T, const Sources& S, i64 n_seg,
                  const int* seg_leaf, const longlong2* seg_range, const i64* seg_out,
                  const i64* partners, const double* la, const double* lb, int order, int width,
                  double eps2, double* partial, double* phi, double* field, i64* status,
                  cudaStream_t s) {
    if (kernel == TD3_KERNEL_LOG)
        return with_potential
                   ? launch_near<TD3_KERNEL_LOG, true, OTHER, LOCAL>(T, S, n_seg, seg_leaf, seg_range,
                                                                      seg_out, partners, la, lb, order,
                                                                      width, eps2, partial, phi,
                                                                      field, status, s)
                   : launch_near<TD3_KERNEL_LOG, false, OTHER, LOCAL>(T, S, n_seg, seg_leaf, seg_range,
                                                                       seg_out, partners, la, lb,
                                                                       order, width, eps2, partial,
                                                                       phi, field, status, s);
    return with_potential
               ? launch_near<TD3_KERNEL_COULOMB, true, OTHER, LOCAL>(T, S, n_seg, seg_leaf, seg_range,
                                                                      seg_out, partners, la, lb,
                                                                      order, width, eps2, partial,
                                                                      phi, field, status, s)
               : launch_near<TD3_KERNEL_COULOMB, false, OTHER, LOCAL>(T, S, n_seg, seg_leaf,
                                                                       seg_range, seg_out, partners,
                                                                       la, lb, order, width, eps2,
                                                                       partial, phi, field, status,
                                                                       s);
}

}  // namespace

extern "C" size_t td3_nearfield_plan_workspace_size(int64_t n_nodes) {
    return 4 * td3_ws_bytes<i64>(n_nodes + 1) + td3_scan_workspace(n_nodes + 1);
}

extern "C" int td3_nearfield_plan(const int64_t* rows, int64_t n_nodes, const int64_t* node_child,
                                  const int64_t* node_start, const int64_t* node_end,
                                  int segment, int* seg_leaf, int64_t* seg_range,
                                  int64_t* seg_out, int64_t seg_capacity, int64_t* sizes,
                                  void* workspace, size_t workspace_bytes, void* stream) {
    if (n_nodes < 1 || segment < 1 || seg_capacity < 0 || n_nodes > 0x7fffffffLL) return TD3_EINVAL;
    cudaStream_t s = td3_stream(stream);
    Workspace w(workspace, workspace_bytes);
    i64* nseg = w.take<i64>(n_nodes + 1);
    i64* psize = w.take<i64>(n_nodes + 1);
    i64* nseg_scan = w.take<i64>(n_nodes + 1);
    i64* psize_scan = w.take<i64>(n_nodes + 1);
    if (!psize_scan) return TD3_EWORKSPACE;
    unsigned nb = td3_blocks(n_nodes, 256);
    k_plan_count<<<nb, 256, 0, s>>>(n_nodes, rows, node_child, node_start, node_end, segment, nseg,
                                    psize);
    TD3_CHECK_LAUNCH();
    TD3_TRY(cudaMemsetAsync(nseg + n_nodes, 0, sizeof(i64), s));
    TD3_TRY(cudaMemsetAsync(psize + n_nodes, 0, sizeof(i64), s));
    TD3_TRY_RC(td3_exclusive_scan_i64(nseg, nseg_scan, n_nodes + 1, nullptr, w.base + w.used,
                                      w.size - w.used, s));
    TD3_TRY_RC(td3_exclusive_scan_i64(psize, psize_scan, n_nodes + 1, nullptr, w.base + w.used,
                                      w.size - w.used, s));
    i64 totals[2];
    TD3_TRY(cudaMemcpyAsync(&totals[0], nseg_scan + n_nodes, sizeof(i64), cudaMemcpyDeviceToHost, s));
    TD3_TRY(cudaMemcpyAsync(&totals[1], psize_scan + n_nodes, sizeof(i64), cudaMemcpyDeviceToHost, s));
    TD3_TRY(cudaStreamSynchronize(s));
    sizes[0] = totals[0];
    sizes[1] = totals[1];
    if (totals[0] > seg_capacity) return TD3_ENEEDMORE;
    k_plan_fill<<<nb, 256, 0, s>>>(n_nodes, rows, node_start, node_end, segment, nseg_scan,
                                   psize_scan, nseg, seg_leaf, reinterpret_cast<longlong2*>(seg_range),
                                   seg_out);
    TD3_CHECK_LAUNCH();
    return TD3_OK;
}

extern "C" int td3_fmm_evaluate(int kernel, const double* sorted_pos, const double* sorted_charge,
                                const int64_t* perm, int64_t n, const double* node_center,
                                const int64_t* node_start, const int64_t* node_end, int order,
                                const double* local_a, const double* local_b,
                                const int64_t* p2p_partners, const int* seg_leaf,
                                const int64_t* seg_range, const int64_t* seg_out, int64_t n_seg,
                                double* partial, double softening, int with_potential,
                                double* phi, double* field, int64_t* status, void* stream) {
    if (n < 0 || n_seg < 0 || order < 0 || order > TD3_MAX_ORDER) return TD3_EINVAL;
    if (kernel != TD3_KERNEL_COULOMB && kernel != TD3_KERNEL_LOG) return TD3_EINVAL;
    if (n == 0) return TD3_OK;
    Targets T{sorted_pos, nullptr, perm, node_center, node_start, node_end, n};
    Sources S{sorted_pos, sorted_charge, perm, node_start, node_end, n};
    double eps2 = softening * softening;
    cudaStream_t s = td3_stream(stream);
    const longlong2* sr = reinterpret_cast<const longlong2*>(seg_range);
    if (kernel == TD3_KERNEL_LOG)
        return dispatch_near<false, LOCAL_COMPLEX>(kernel, with_potential, T, S, n_seg, seg_leaf, sr,
                                                   seg_out, p2p_partners, local_a, local_b, order,
                                                   order + 1, eps2, partial, phi, field, status, s);
    return dispatch_near<false, LOCAL_CART>(kernel, with_potential, T, S, n_seg, seg_leaf, sr,
                                            seg_out, p2p_partners, local_a, local_b, order,
                                            (order + 1) * (order + 2) / 2, eps2, partial, phi, field,
                                            status, s);
}

extern "C" int td3_fmm_targets(int kernel, const double* sorted_targets,
                               const int64_t* sorted_exclude, const int64_t* target_perm,
                               int64_t m, const double* t_center, const int64_t* t_start,
                               const int64_t* t_end, int order, const double* local_a,
                               const double* local_b, const int64_t* p2p_partners,
                               const int* seg_leaf, const int64_t* seg_range,
                               const int64_t* seg_out, int64_t n_seg, double* partial,
                               const double* sorted_pos, const double* sorted_charge,
                               const int64_t* perm, int64_t n, const int64_t* s_start,
                               const int64_t* s_end, double softening, int with_potential,
                               double* phi, double* field, int64_t* status, void* stream) {
    if (m < 0 || n < 0 || n_seg < 0 || order < 0 || order > TD3_MAX_ORDER) return TD3_EINVAL;
    if (kernel != TD3_KERNEL_COULOMB && kernel != TD3_KERNEL_LOG) return TD3_EINVAL;
    if (m == 0) return TD3_OK;
    Targets T{sorted_targets, sorted_exclude, target_perm, t_center, t_start, t_end, m};
    Sources S{sorted_pos, sorted_charge, perm, s_start, s_end, n};
    double eps2 = softening * softening;
    cudaStream_t s = td3_stream(stream);
    const longlong2* sr = reinterpret_cast<const longlong2*>(seg_range);
    if (kernel == TD3_KERNEL_LOG)
        return dispatch_near<true, LOCAL_COMPLEX>(kernel, with_potential, T, S, n_seg, seg_leaf, sr,
                                                  seg_out, p2p_partners, local_a, local_b, order,
                                                  order + 1, eps2, partial, phi, field, status, s);
    return dispatch_near<true, LOCAL_CART>(kernel, with_potential, T, S, n_seg, seg_leaf, sr,
                                           seg_out, p2p_partners, local_a, local_b, order,
                                           (order + 1) * (order + 2) / 2, eps2, partial, phi, field,
                                           status, s);
}
