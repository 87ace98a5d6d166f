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

constexpr int NF_WARPS = 4;   // warps per block of the finish kernels
// Warps per block of the one-launch pair kernels (k_near, k_near_adjoint): one, so a
// segment's warp frees its slot when it ends rather than with its block's slowest segment.
constexpr int NW_NEAR = 1;
constexpr int LOCAL_COMPLEX = 0;
constexpr int LOCAL_CART = 1;

// Blocks of a finish launch: a warp per 32 segments, at most 148 x 16 blocks.
static inline unsigned td3_finish_blocks(i64 n_seg) {
    const i64 warps = (n_seg + 31) / 32, blocks = (warps + NF_WARPS - 1) / NF_WARPS;
    return (unsigned)(blocks < 1 ? 1 : blocks > 148 * 16 ? 148 * 16 : blocks);
}

__device__ __forceinline__ int pow2_at_least(int v) {
    int p = 1;
    while (p < v) p <<= 1;
    return p;
}

// ------------------------------------------------------------------ the plan
__global__ void k_plan_count(i64 n_nodes, const i64* __restrict__ rows, const i64* __restrict__ child,
                             const i64* __restrict__ start, const i64* __restrict__ end, int segment,
                             i64* __restrict__ nseg, i64* __restrict__ psize) {
    td3_chain_wait();
    td3_chain_release();
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
    td3_chain_wait();
    td3_chain_release();
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

// Value, gradient and Hessian of the potential of a local expansion at u = r - c:
// log kernel phi = -2 Re W (W = sum b_l u^l), Coulomb phi = sum T_(a,b) ux^a uy^b.
struct LocalJet {
    double v, gx, gy, hxx, hxy, hyy;
};

__device__ __forceinline__ LocalJet jet_complex(const double* __restrict__ lre,
                                                const double* __restrict__ lim, int order,
                                                double ux, double uy) {
    double wr = lre[order], wi = lim[order], d1r = 0.0, d1i = 0.0, d2r = 0.0, d2i = 0.0;
    for (int l = order - 1; l >= 0; --l) {
        double t;
        t = d2r * ux - d2i * uy + d1r;
        d2i = d2r * uy + d2i * ux + d1i;
        d2r = t;
        t = d1r * ux - d1i * uy + wr;
        d1i = d1r * uy + d1i * ux + wi;
        d1r = t;
        t = wr * ux - wi * uy + lre[l];
        wi = wr * uy + wi * ux + lim[l];
        wr = t;
    }
    // W'' = 2 d2
    return {-2.0 * wr, -2.0 * d1r, 2.0 * d1i, -4.0 * d2r, 4.0 * d2i, 4.0 * d2r};
}

__device__ __forceinline__ LocalJet jet_cart(const double* __restrict__ T, int order, double ux,
                                             double uy) {
    // outer Horner in uy over P_b(ux) and its x-derivatives, inner Horner in ux
    double q = 0.0, qy = 0.0, qyy = 0.0, gx = 0.0, gxy = 0.0, k = 0.0;
    for (int b = order; b >= 0; --b) {
        int top = order - b;
        int n = top + b;
        double p = T[n * (n + 1) / 2 + b], p1 = 0.0, p2 = 0.0;
        for (int a = top - 1; a >= 0; --a) {
            n = a + b;
            p2 = p2 * ux + p1;
            p1 = p1 * ux + p;
            p = p * ux + T[n * (n + 1) / 2 + b];
        }
        qyy = qyy * uy + qy;
        qy = qy * uy + q;
        q = q * uy + p;
        gxy = gxy * uy + gx;
        gx = gx * uy + p1;
        k = k * uy + 2.0 * p2;
    }
    return {q, gx, qy, k, gxy, 2.0 * qyy};
}

template <int LOCAL>
__device__ __forceinline__ LocalJet local_jet(const double* __restrict__ la,
                                              const double* __restrict__ lb, i64 leaf, int order,
                                              int width, double ux, double uy) {
    if (LOCAL == LOCAL_COMPLEX) return jet_complex(la + leaf * width, lb + leaf * width, order, ux, uy);
    return jet_cart(la + leaf * width, order, ux, uy);
}

struct Sources {
    const double* pos;     // (2, n) tree order
    const double* charge;  // (n) tree order
    const i64* index;      // (n) input index of each slot (exclusion)
    const i64* start;
    const i64* end;
    i64 n;
    double unit;  // length unit L of the mixed-precision pair arithmetic
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

// ------------------------------------------------------------------ staged sources
// The source particles of a segment's partner leaves pass through shared memory: the
// warp takes 32 partner leaves at a time (lane i reads leaf i's range; a warp scan of
// the counts places them), copies their particles in windows of up to CAP (every lane
// loads independent particles, so the loads overlap), and then every (target, slice)
// lane sums over the window.  Each target still meets every source once, in a fixed
// order (window by window, slice-strided inside a window, slices added last).
//
// stage(p, j): store source slot j at window position p (called by one lane);
// body(wn): sum over the window's wn staged particles (called by every lane).
template <int CAP, class Stage, class Body>
__device__ __forceinline__ void for_source_windows(const Sources& S,
                                                   const i64* __restrict__ partners, i64 e0,
                                                   i64 e1, int lane, Stage stage, Body body) {
    for (i64 g = e0; g < e1; g += 32) {
        i64 i = g + lane;
        i64 st = 0;
        int cnt = 0;
        if (i < e1) {
            i64 b = partners[i];
            st = S.start[b];
            cnt = (int)(S.end[b] - st);
        }
        int incl = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        int total = __shfl_sync(0xffffffffu, incl, 31);
        int excl = incl - cnt;
        for (int w0 = 0; w0 < total; w0 += CAP) {
            int wn = total - w0 < CAP ? total - w0 : CAP;
            for (int p0 = 0; p0 < wn; p0 += 32) {
                int p = p0 + lane;
                int at = w0 + (p < wn ? p : 0);
                // the leaf holding position `at`: the last lane whose offset is <= at
                int L = 0;
#pragma unroll
                for (int s = 16; s > 0; s >>= 1) {
                    int v = __shfl_sync(0xffffffffu, excl, L + s);
                    if (v <= at) L += s;
                }
                i64 stL = __shfl_sync(0xffffffffu, st, L);
                int exL = __shfl_sync(0xffffffffu, excl, L);
                if (p < wn) stage(p, stL + (at - exL));
            }
            __syncwarp();
            body(wn);
            __syncwarp();
        }
    }
}

constexpr int NF_CAP = 256;  // staged sources per warp window (forward)

struct NearWindow {
    double x[NF_CAP], y[NF_CAP], q[NF_CAP];
    int tag[NF_CAP];  // slot j (self-exclusion) or the source's input index (OTHER)
};

// The length unit u of the mixed-precision pair arithmetic: the power of two with
// unit <= u < 2 unit.  Positions scale by 1/u exactly, so the FP64 difference of two
// scaled positions is the scaled FP64 difference of the positions.
__device__ __forceinline__ double pair_unit(double unit) {
    int e;
    frexp(unit, &e);
    return ldexp(1.0, e);
}

// One mixed-precision pair: the difference in FP64 (exact enough for close pairs far
// from the origin), in units of L = S.unit and rounded to FP32, then FP32 arithmetic with
// compensated accumulation.  Coulomb sums q / r' and q d' / r'^3; log sums -q ln r'^2
// (with the charges in FP64, qsum) and 2 q d' / r'^2.
template <int KERNEL, bool POT>
__device__ __forceinline__ void pair_mixed(double dx64, double dy64, double qj, double inv_unit,
                                           float eps2f, float& p, float& x, float& y,
                                           double& qsum) {
    float dx = (float)(dx64 * inv_unit), dy = (float)(dy64 * inv_unit), q = (float)qj;
    float r2 = dx * dx + dy * dy + eps2f;
    if (KERNEL == TD3_KERNEL_LOG) {
        if (POT) {
            p += -q * __logf(r2);
            qsum += qj;
        }
        float f = __fdividef(2.0f * q, r2);
        x += f * dx;
        y += f * dy;
    } else {
        float inv_r = rsqrtf(r2);
        float qr3 = q * inv_r * inv_r * inv_r;
        p += q * inv_r;
        x += qr3 * dx;
        y += qr3 * dy;
    }
}

// Pairs summed in plain FP32 before one compensated addition: each lane adds the terms
// of NF_BLOCK consecutive pairs of its slice, then the block's sum to the compensated
// accumulator (the rounding of a 16-term sum, then compensated across blocks).
constexpr int NF_BLOCK = 16;

// One warp per segment.  OTHER: targets and sources are different point sets (fmm_at):
// zero charges and source exclude[i] are skipped and any coincidence is an error.
// Otherwise targets are the sources themselves: a particle skips itself and a
// coincident pair is an error only if both charges are nonzero.  MIXED: FP32 pair
// arithmetic with compensated sums (pair_mixed), else FP64.  The sources come through
// shared memory (for_source_windows).
template <int KERNEL, bool POT, bool OTHER, int LOCAL, bool MIXED>
__global__ void __launch_bounds__(32 * NW_NEAR, 28 / NW_NEAR)
k_near(Targets T, Sources S, i64 n_seg, const int* __restrict__ seg_leaf,
       const longlong2* __restrict__ seg_range, const i64* __restrict__ seg_out,
       const i64* __restrict__ partners, const double* __restrict__ local_a,
       const double* __restrict__ local_b, int order, int width, double eps2,
       double* __restrict__ partial, double* __restrict__ phi, double* __restrict__ field,
       i64* status) {
    td3_chain_wait();
    td3_chain_release();
    __shared__ NearWindow windows[NW_NEAR];
    int lane = threadIdx.x & 31;
    NearWindow& win = windows[threadIdx.x >> 5];
    i64 seg = (i64)blockIdx.x * NW_NEAR + (threadIdx.x >> 5);
    if (seg >= n_seg) return;
    i64 leaf = seg_leaf[seg];
    longlong2 er = seg_range[seg];
    i64 outp = seg_out[seg];
    i64 s0 = T.start[leaf];
    int count = (int)(T.end[leaf] - s0);
    int tsz = pow2_at_least(count < 32 ? count : 32);
    int slices = 32 / tsz;
    int ti = lane % tsz, slice = lane / tsz;
    const double inv_unit = 1.0 / S.unit;
    const float eps2f = (float)(eps2 * inv_unit * inv_unit);
    auto stage = [&](int p, i64 j) {
        win.x[p] = S.pos[j];
        win.y[p] = S.pos[S.n + j];
        win.q[p] = S.charge[j];
        win.tag[p] = OTHER ? (int)S.index[j] : (int)j;
    };
    for (int base = 0; base < count; base += tsz) {
        int it = base + ti;
        bool valid = it < count;
        i64 k = s0 + (valid ? it : 0);
        double xi = T.pos[k], yi = T.pos[T.m + k];
        double qi = OTHER ? 0.0 : S.charge[k];
        i64 skip = OTHER ? (T.exclude ? T.exclude[k] : -1) : k;
        double pot = 0.0, ex = 0.0, ey = 0.0;
        bool bad = false;
        KahanF kp, kx, ky;
        double qsum = 0.0;
        for_source_windows<NF_CAP>(S, partners, er.x, er.y, lane, stage, [&](int wn) {
            if (!valid) return;
            if constexpr (MIXED) {
                for (int p0 = slice; p0 < wn; p0 += NF_BLOCK * slices) {
                    float bp = 0.0f, bx = 0.0f, by = 0.0f;
                    int p1 = p0 + NF_BLOCK * slices < wn ? p0 + NF_BLOCK * slices : wn;
                    for (int p = p0; p < p1; p += slices) {
                        double qj = win.q[p];
                        i64 tag = win.tag[p];
                        if (OTHER) {
                            if (qj == 0.0 || tag == skip) continue;
                        } else if (tag == skip) {
                            continue;
                        }
                        double dx = xi - win.x[p], dy = yi - win.y[p];
                        if (dx == 0.0 && dy == 0.0 && eps2 == 0.0) {
                            bad |= OTHER ? true : (qi != 0.0 && qj != 0.0);
                            continue;
                        }
                        pair_mixed<KERNEL, POT>(dx, dy, qj, inv_unit, eps2f, bp, bx, by, qsum);
                    }
                    if (POT || KERNEL != TD3_KERNEL_LOG) kp.add(bp);
                    kx.add(bx);
                    ky.add(by);
                }
            } else {
                for (int p = slice; p < wn; p += slices) {
                    double qj = win.q[p];
                    i64 tag = win.tag[p];
                    if (OTHER) {
                        if (qj == 0.0 || tag == skip) continue;
                    } else if (tag == skip) {
                        continue;
                    }
                    double dx = xi - win.x[p], dy = yi - win.y[p];
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
        });
        if (MIXED) {
            // back from units of L: Coulomb 1/L, 1/L^2; log -ln L^2 sum q, 1/L
            if (KERNEL == TD3_KERNEL_LOG) {
                pot = kp.value() - 2.0 * log(S.unit) * qsum;
                ex = kx.value() * inv_unit;
                ey = ky.value() * inv_unit;
            } else {
                pot = kp.value() * inv_unit;
                ex = kx.value() * inv_unit * inv_unit;
                ey = ky.value() * inv_unit * inv_unit;
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

// The number of consecutive segments of `leaf` starting at its first segment `seg`,
// found 32 segments at a time (the same value in every lane).
__device__ __forceinline__ i64 leaf_segments(const int* __restrict__ seg_leaf, i64 seg, i64 n_seg,
                                             i64 leaf, int lane) {
    i64 count = 0;
    for (;;) {
        i64 s = seg + count + lane;
        bool same = s < n_seg && seg_leaf[s] == leaf;
        unsigned m = __ballot_sync(0xffffffffu, same);
        if (m == 0xffffffffu) {
            count += 32;
            continue;
        }
        return count + __ffs(~m) - 1;
    }
}

// One multi-segment leaf (its first segment `seg`): every target's partial sums over the
// segments, then L2P (or, ADD, written alone for k_far_field to complete).
template <bool POT, int LOCAL, bool ADD>
__device__ __forceinline__ void finish_leaf(Targets T, i64 n_seg, const int* __restrict__ seg_leaf,
                                            const i64* __restrict__ seg_out,
                                            const double* __restrict__ local_a,
                                            const double* __restrict__ local_b, int order,
                                            int width, const double* __restrict__ partial,
                                            double* __restrict__ phi, double* __restrict__ field,
                                            i64 seg, int lane) {
    i64 leaf = seg_leaf[seg];
    i64 s0 = T.start[leaf];
    int count = (int)(T.end[leaf] - s0);
    i64 nseg = leaf_segments(seg_leaf, seg, n_seg, leaf, lane);
    // the partial sums of a target over the leaf's segments: lanes split the segments
    // (a row can take thousands), a fixed-order warp reduction combines them
    for (int it = 0; it < count; ++it) {
        double pot = 0.0, ex = 0.0, ey = 0.0;
        for (i64 s = seg + lane; s < seg + nseg; s += 32) {
            i64 p = seg_out[s] + it;
            pot += partial[3 * p];
            ex += partial[3 * p + 1];
            ey += partial[3 * p + 2];
        }
        for (int off = 16; off > 0; off >>= 1) {
            pot += __shfl_xor_sync(0xffffffffu, pot, off);
            ex += __shfl_xor_sync(0xffffffffu, ex, off);
            ey += __shfl_xor_sync(0xffffffffu, ey, off);
        }
        if (ADD && lane == (it & 31)) {
            const i64 i = T.perm[s0 + it];
            phi[i] = POT ? pot : 0.0;
            field[i] = ex;
            field[T.m + i] = ey;
        } else if (lane == (it & 31)) {
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
}

// Leaves whose row took several segments: partial sums in segment order, plus L2P (or,
// ADD, the near sums alone, which k_far_field completes).  Launched over a fraction of the
// segments' warps (td3_finish_blocks): most leaves have one segment.
template <bool POT, int LOCAL, bool ADD = false>
__global__ void k_near_finish(Targets T, i64 n_seg, const int* __restrict__ seg_leaf,
                              const i64* __restrict__ seg_out, const double* __restrict__ local_a,
                              const double* __restrict__ local_b, int order, int width,
                              const double* __restrict__ partial, double* __restrict__ phi,
                              double* __restrict__ field) {
    td3_chain_wait();
    td3_chain_release();
    const int lane = threadIdx.x & 31;
    // the first segment of a multi-segment leaf finishes it; each warp scans 32 segments
    // at a time for them
    const i64 warps = (i64)gridDim.x * NF_WARPS;
    for (i64 base = ((i64)blockIdx.x * NF_WARPS + (threadIdx.x >> 5)) * 32; base < n_seg;
         base += warps * 32) {
        const i64 mine = base + lane;
        unsigned firsts = __ballot_sync(
            0xffffffffu, mine < n_seg && seg_out[mine] >= 0 &&
                             (mine == 0 || seg_leaf[mine - 1] != seg_leaf[mine]));
        while (firsts) {
            const i64 seg = base + __ffs(firsts) - 1;
            firsts &= firsts - 1;
            finish_leaf<POT, LOCAL, ADD>(T, n_seg, seg_leaf, seg_out, local_a, local_b, order,
                                         width, partial, phi, field, seg, lane);
        }
    }
}

// ------------------------------------------------------------------ adjoint pass
// Backward of (phi, E) at the sources for upstream gradients (w = dL/dphi, e = dL/dE):
//   dL/dq_k = Psi(x_k),  dL/dx_k = -w_k E_k + q_k grad Psi(x_k) - M_k e_k,
// Psi(y) = sum_j [w_j G(y - x_j) + e_j . grad G(y - x_j)] (monopoles w and dipoles e at
// the sources, j != k), M_k = sum_j q_j Hess G(x_k - x_j) (the Hessian of the forward
// potential).  Near parts are summed here pair by pair; the far parts come from the
// adjoint pass's local expansion (value and gradient) and the forward one (Hessian).
struct Adjoint {
    const double* weight;  // (n) w in tree order
    const double* dipole;  // (2, n) e in tree order
    const double* efield;  // (2, n) forward E, input order
    double* qbar;          // (n) input order
    double* xbar;          // (2, n) input order
};

template <int KERNEL>
__device__ __forceinline__ void adjoint_pair(double dx, double dy, double eps2, double qj,
                                             double wj, double exj, double eyj, double* acc) {
    double s = dx * dx + dy * dy + eps2;
    double de = exj * dx + eyj * dy;
    if (KERNEL == TD3_KERNEL_LOG) {
        // G = -ln s, grad G = -2 d / s, Hess G = -2 I / s + 4 d d^T / s^2
        double inv = 1.0 / s;
        double lg = log(s);
        acc[0] += -wj * lg - 2.0 * de * inv;
        double t = 4.0 * de * inv * inv;
        acc[1] += -2.0 * inv * (wj * dx + exj) + t * dx;
        acc[2] += -2.0 * inv * (wj * dy + eyj) + t * dy;
        double q4 = 4.0 * qj * inv * inv;
        acc[3] += -2.0 * qj * inv + q4 * dx * dx;
        acc[4] += q4 * dx * dy;
        acc[5] += -2.0 * qj * inv + q4 * dy * dy;
    } else {
        // G = s^(-1/2), grad G = -d s^(-3/2), Hess G = -I s^(-3/2) + 3 d d^T s^(-5/2)
        double r = rsqrt(s);
        double r3 = r * r * r;
        double r5 = r3 * r * r;
        acc[0] += wj * r - de * r3;
        double t = 3.0 * de * r5;
        acc[1] += -r3 * (wj * dx + exj) + t * dx;
        acc[2] += -r3 * (wj * dy + eyj) + t * dy;
        double q3 = 3.0 * qj * r5;
        acc[3] += -qj * r3 + q3 * dx * dx;
        acc[4] += q3 * dx * dy;
        acc[5] += -qj * r3 + q3 * dy * dy;
    }
}

// adjoint_pair in FP32 with compensated accumulators (the pair difference arrives in FP32
// after an FP64 subtraction).
template <int KERNEL>
__device__ __forceinline__ void adjoint_pair_mixed(float dx, float dy, float eps2, float qj,
                                                   float wj, float exj, float eyj, float* acc) {
    float s = dx * dx + dy * dy + eps2;
    float de = exj * dx + eyj * dy;
    if (KERNEL == TD3_KERNEL_LOG) {
        float inv = __frcp_rn(s);
        acc[0] += -wj * __logf(s) - 2.0f * de * inv;
        float t = 4.0f * de * inv * inv;
        acc[1] += -2.0f * inv * (wj * dx + exj) + t * dx;
        acc[2] += -2.0f * inv * (wj * dy + eyj) + t * dy;
        float q4 = 4.0f * qj * inv * inv;
        acc[3] += -2.0f * qj * inv + q4 * dx * dx;
        acc[4] += q4 * dx * dy;
        acc[5] += -2.0f * qj * inv + q4 * dy * dy;
    } else {
        float r = rsqrtf(s);
        float r3 = r * r * r;
        float r5 = r3 * r * r;
        acc[0] += wj * r - de * r3;
        float t = 3.0f * de * r5;
        acc[1] += -r3 * (wj * dx + exj) + t * dx;
        acc[2] += -r3 * (wj * dy + eyj) + t * dy;
        float q3 = 3.0f * qj * r5;
        acc[3] += -qj * r3 + q3 * dx * dx;
        acc[4] += q3 * dx * dy;
        acc[5] += -qj * r3 + q3 * dy * dy;
    }
}

// qbar and xbar of slot k (input index i) from the near sums acc and the far parts: f
// the forward local expansion's jet (its Hessian), b the adjoint one's (Psi, grad Psi).
__device__ __forceinline__ void adjoint_combine(const double* acc, const LocalJet& f,
                                                const LocalJet& b, i64 k, i64 i, i64 n,
                                                const Sources& S, const Adjoint& A) {
    double psi = acc[0] + b.v;
    double gx = acc[1] + b.gx, gy = acc[2] + b.gy;
    double mxx = acc[3] + f.hxx, mxy = acc[4] + f.hxy, myy = acc[5] + f.hyy;
    double q = S.charge[k], w = A.weight[k], ex = A.dipole[k], ey = A.dipole[n + k];
    A.qbar[i] = psi;
    A.xbar[i] = -w * A.efield[i] + q * gx - (mxx * ex + mxy * ey);
    A.xbar[n + i] = -w * A.efield[n + i] + q * gy - (mxy * ex + myy * ey);
}

// The near part of qbar and xbar of slot k (input index i), written alone; k_far_adjoint
// adds the far part (qbar and xbar are linear in the near sums acc).
__device__ __forceinline__ void adjoint_add(const double* acc, i64 k, i64 i, i64 n,
                                            const Sources& S, const Adjoint& A) {
    const double q = S.charge[k], ex = A.dipole[k], ey = A.dipole[n + k];
    A.qbar[i] = acc[0];
    A.xbar[i] = q * acc[1] - (acc[3] * ex + acc[4] * ey);
    A.xbar[n + i] = q * acc[2] - (acc[4] * ex + acc[5] * ey);
}

// The far part of qbar and xbar of slot k (input index i) added to the near part: f the
// forward local expansion's jet (its Hessian), b the adjoint one's (Psi, grad Psi).
__device__ __forceinline__ void adjoint_far_add(const LocalJet& f, const LocalJet& b, i64 k, i64 i,
                                                i64 n, const Sources& S, const Adjoint& A) {
    const double q = S.charge[k], w = A.weight[k], ex = A.dipole[k], ey = A.dipole[n + k];
    A.qbar[i] += b.v;
    A.xbar[i] += -w * A.efield[i] + q * b.gx - (f.hxx * ex + f.hxy * ey);
    A.xbar[n + i] += -w * A.efield[n + i] + q * b.gy - (f.hxy * ex + f.hyy * ey);
}

template <int LOCAL>
__device__ __forceinline__ void adjoint_finish(const double* acc, i64 k, i64 i, i64 n,
                                               double ux, double uy, i64 leaf, int order,
                                               int width, const double* fa, const double* fb,
                                               const double* ba, const double* bb,
                                               const Sources& S, const Adjoint& A) {
    LocalJet f = local_jet<LOCAL>(fa, fb, leaf, order, width, ux, uy);  // forward: Hessian
    LocalJet b = local_jet<LOCAL>(ba, bb, leaf, order, width, ux, uy);  // adjoint: Psi
    adjoint_combine(acc, f, b, k, i, n, S, A);
}

constexpr int NF_CAP_ADJ = 128;  // staged sources per warp window (adjoint)

// FP64: positions, charges, monopoles and dipoles.  Mixed: positions (scaled by 1/u)
// and monopoles in FP64 (the pair difference and the monopole sum), the rest in FP32
// (dipoles scaled by 1/u), converted once per staged source instead of once per pair.
template <bool MIXED>
struct AdjointWindow {
    double x[NF_CAP_ADJ], y[NF_CAP_ADJ], q[NF_CAP_ADJ], w[NF_CAP_ADJ], ex[NF_CAP_ADJ],
        ey[NF_CAP_ADJ];
    int tag[NF_CAP_ADJ];  // slot j (self-exclusion)
};
template <>
struct AdjointWindow<true> {
    double x[NF_CAP_ADJ], y[NF_CAP_ADJ], w[NF_CAP_ADJ];
    float qf[NF_CAP_ADJ], wf[NF_CAP_ADJ], exf[NF_CAP_ADJ], eyf[NF_CAP_ADJ];
    int tag[NF_CAP_ADJ];
};

template <int KERNEL, int LOCAL, bool MIXED>
__global__ void __launch_bounds__(32 * NW_NEAR, 24 / NW_NEAR)
k_near_adjoint(Targets T, Sources S, Adjoint A, i64 n_seg, const int* __restrict__ seg_leaf,
               const longlong2* __restrict__ seg_range, const i64* __restrict__ seg_out,
               const i64* __restrict__ partners, const double* __restrict__ fa,
               const double* __restrict__ fb, const double* __restrict__ ba,
               const double* __restrict__ bb, int order, int width, double eps2,
               double* __restrict__ partial) {
    td3_chain_wait();
    td3_chain_release();
    __shared__ AdjointWindow<MIXED> windows[NW_NEAR];
    int lane = threadIdx.x & 31;
    AdjointWindow<MIXED>& win = windows[threadIdx.x >> 5];
    i64 seg = (i64)blockIdx.x * NW_NEAR + (threadIdx.x >> 5);
    if (seg >= n_seg) return;
    i64 leaf = seg_leaf[seg];
    longlong2 er = seg_range[seg];
    i64 outp = seg_out[seg];
    i64 s0 = T.start[leaf];
    int count = (int)(T.end[leaf] - s0);
    int tsz = pow2_at_least(count < 32 ? count : 32);
    int slices = 32 / tsz;
    int ti = lane % tsz, slice = lane / tsz;
    i64 n = S.n;
    // mixed: in units of L = S.unit (d' = d / L, e' = e / L) the log kernel's sums scale
    // as (1, 1/L, 1/L^2) plus -ln L^2 sum w for Psi, the Coulomb kernel's as
    // (1/L, 1/L^2, 1/L^3)
    // mixed: positions in units of u (pair_unit), scaled exactly
    const double unit = MIXED ? pair_unit(S.unit) : 1.0, inv_unit = 1.0 / unit;
    const float eps2f = (float)(eps2 * inv_unit * inv_unit);
    auto stage = [&](int p, i64 j) {
        win.x[p] = S.pos[j] * inv_unit;
        win.y[p] = S.pos[n + j] * inv_unit;
        win.w[p] = A.weight[j];
        win.tag[p] = (int)j;
        if constexpr (MIXED) {
            win.qf[p] = (float)S.charge[j];
            win.wf[p] = (float)A.weight[j];
            win.exf[p] = (float)(A.dipole[j] * inv_unit);
            win.eyf[p] = (float)(A.dipole[n + j] * inv_unit);
        } else {
            win.q[p] = S.charge[j];
            win.ex[p] = A.dipole[j];
            win.ey[p] = A.dipole[n + j];
        }
    };
    for (int base = 0; base < count; base += tsz) {
        int it = base + ti;
        bool valid = it < count;
        i64 k = s0 + (valid ? it : 0);
        double xi = S.pos[k], yi = S.pos[n + k];
        double xs = xi * inv_unit, ys = yi * inv_unit;
        int self = (int)k;
        double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        KahanF kacc[6];
        double wsum = 0.0;
        for_source_windows<NF_CAP_ADJ>(S, partners, er.x, er.y, lane, stage, [&](int wn) {
            if (!valid) return;
            if constexpr (MIXED) {
                for (int p0 = slice; p0 < wn; p0 += NF_BLOCK * slices) {
                    float blk[6] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
                    int p1 = p0 + NF_BLOCK * slices < wn ? p0 + NF_BLOCK * slices : wn;
                    for (int p = p0; p < p1; p += slices) {
                        if (win.tag[p] == self) continue;
                        double dx = xs - win.x[p], dy = ys - win.y[p];
                        float dxf = (float)dx, dyf = (float)dy;
                        if (dxf == 0.0f && dyf == 0.0f && eps2 == 0.0 && dx == 0.0 && dy == 0.0)
                            continue;
                        if (KERNEL == TD3_KERNEL_LOG) wsum += win.w[p];
                        adjoint_pair_mixed<KERNEL>(dxf, dyf, eps2f, win.qf[p], win.wf[p],
                                                   win.exf[p], win.eyf[p], blk);
                    }
#pragma unroll
                    for (int c = 0; c < 6; ++c) kacc[c].add(blk[c]);
                }
            } else {
                for (int p = slice; p < wn; p += slices) {
                    if (win.tag[p] == self) continue;
                    double dx = xs - win.x[p], dy = ys - win.y[p];
                    if (dx * dx + dy * dy + eps2 == 0.0) continue;
                    adjoint_pair<KERNEL>(dx, dy, eps2, win.q[p], win.w[p], win.ex[p], win.ey[p],
                                         acc);
                }
            }
        });
        if (MIXED) {
            double sc = KERNEL == TD3_KERNEL_LOG ? 1.0 : inv_unit;
            acc[0] = kacc[0].value() * sc;
            if (KERNEL == TD3_KERNEL_LOG) acc[0] -= 2.0 * log(unit) * wsum;
            for (int c = 1; c < 3; ++c) acc[c] = kacc[c].value() * (sc * inv_unit);
            for (int c = 3; c < 6; ++c) acc[c] = kacc[c].value() * (sc * inv_unit * inv_unit);
        }
#pragma unroll
        for (int c = 0; c < 6; ++c)
            for (int off = tsz; off < 32; off <<= 1)
                acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], off);
        if (outp < 0) {
            // the two far-field jets in one instruction stream: slice 0 evaluates the
            // forward expansion, slice 1 the adjoint one (with a single slice, slice 0
            // evaluates both)
            double ux = xi - T.center[2 * leaf], uy = yi - T.center[2 * leaf + 1];
            bool adj = slices > 1 && slice == 1;
            LocalJet f{}, b{};
            if (valid && slice <= 1)
                f = local_jet<LOCAL>(adj ? ba : fa, adj ? bb : fb, leaf, order, width, ux, uy);
            if (slices > 1) {
                b.v = __shfl_down_sync(0xffffffffu, f.v, tsz);
                b.gx = __shfl_down_sync(0xffffffffu, f.gx, tsz);
                b.gy = __shfl_down_sync(0xffffffffu, f.gy, tsz);
            } else if (valid) {
                b = local_jet<LOCAL>(ba, bb, leaf, order, width, ux, uy);
            }
            if (valid && slice == 0) adjoint_combine(acc, f, b, k, T.perm[k], n, S, A);
        } else if (valid && slice == 0) {
            i64 p = outp + it;
            for (int c = 0; c < 6; ++c) partial[6 * p + c] = acc[c];
        }
    }
}

// One multi-segment leaf of the adjoint pass (its first segment `seg`), as finish_leaf.
template <int LOCAL, bool ADD>
__device__ __forceinline__ void finish_adjoint_leaf(Targets T, Sources S, Adjoint A, i64 n_seg,
                                                    const int* __restrict__ seg_leaf,
                                                    const i64* __restrict__ seg_out,
                                                    const double* __restrict__ fa,
                                                    const double* __restrict__ fb,
                                                    const double* __restrict__ ba,
                                                    const double* __restrict__ bb, int order,
                                                    int width, const double* __restrict__ partial,
                                                    i64 seg, int lane) {
    i64 leaf = seg_leaf[seg];
    i64 s0 = T.start[leaf];
    int count = (int)(T.end[leaf] - s0);
    i64 nseg = leaf_segments(seg_leaf, seg, n_seg, leaf, lane);
    for (int it = 0; it < count; ++it) {
        double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        for (i64 s = seg + lane; s < seg + nseg; s += 32) {
            i64 p = seg_out[s] + it;
            for (int c = 0; c < 6; ++c) acc[c] += partial[6 * p + c];
        }
        for (int c = 0; c < 6; ++c)
            for (int off = 16; off > 0; off >>= 1)
                acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], off);
        if (ADD && lane == (it & 31)) {
            adjoint_add(acc, s0 + it, T.perm[s0 + it], S.n, S, A);
        } else if (lane == (it & 31)) {
            i64 k = s0 + it;
            adjoint_finish<LOCAL>(acc, k, T.perm[k], S.n, S.pos[k] - T.center[2 * leaf],
                                  S.pos[S.n + k] - T.center[2 * leaf + 1], leaf, order, width,
                                  fa, fb, ba, bb, S, A);
        }
    }
}

template <int LOCAL, bool ADD = false>
__global__ void k_near_adjoint_finish(Targets T, Sources S, Adjoint A, i64 n_seg,
                                      const int* __restrict__ seg_leaf,
                                      const i64* __restrict__ seg_out, const double* __restrict__ fa,
                                      const double* __restrict__ fb, const double* __restrict__ ba,
                                      const double* __restrict__ bb, int order, int width,
                                      const double* __restrict__ partial) {
    td3_chain_wait();
    td3_chain_release();
    const int lane = threadIdx.x & 31;
    const i64 warps = (i64)gridDim.x * NF_WARPS;
    for (i64 base = ((i64)blockIdx.x * NF_WARPS + (threadIdx.x >> 5)) * 32; base < n_seg;
         base += warps * 32) {
        const i64 mine = base + lane;
        unsigned firsts = __ballot_sync(
            0xffffffffu, mine < n_seg && seg_out[mine] >= 0 &&
                             (mine == 0 || seg_leaf[mine - 1] != seg_leaf[mine]));
        while (firsts) {
            const i64 seg = base + __ffs(firsts) - 1;
            firsts &= firsts - 1;
            finish_adjoint_leaf<LOCAL, ADD>(T, S, A, n_seg, seg_leaf, seg_out, fa, fb, ba, bb,
                                            order, width, partial, seg, lane);
        }
    }
}

// ------------------------------------------------------------------ mixed form at the sources
// The mixed-precision near field at the sources in two parts: the near part writes the
// pair sums (k_near_mixed / k_near_adjoint_mixed, then the partial sums of the leaves
// that took several segments, k_near_finish / k_near_adjoint_finish with ADD); the far
// part adds the local expansions of every particle in FP64, one thread per slot
// (k_far_field / k_far_adjoint: every lane busy, where a segment's warp would run it on
// one lane per target).  The near part needs no expansion, so a caller can run it on
// another stream while the M2M, M2L and L2L run.
//
// Pair arithmetic: positions relative to the target leaf's centre, in units of the
// power-of-two length u (pair_unit), as FP32 hi + lo pairs (x = hi + lo to 2^-48
// relative); a pair's difference is (hi_i - hi_j) + (lo_i - lo_j), exact in its hi part
// for close pairs, so no FP64 operation is left in the pair loop.  Lanes are (target,
// slice) with floor(32 / targets) slices (no power-of-two rounding); the slices of a
// target are added by a fixed-order tree.

// Slot -> leaf: the leaf holding every particle slot (thread per node).
__global__ void k_slot_leaves(i64 n_nodes, const i64* __restrict__ child,
                              const i64* __restrict__ start, const i64* __restrict__ end,
                              int* __restrict__ slot_leaf) {
    td3_chain_wait();
    td3_chain_release();
    const i64 node = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (node >= n_nodes || child[node] >= 0) return;
    for (i64 k = start[node]; k < end[node]; ++k) slot_leaf[k] = (int)node;
}

template <int LOCAL, bool POT>
__global__ void k_far_field(Targets T, const int* __restrict__ slot_leaf,
                            const double* __restrict__ la, const double* __restrict__ lb,
                            int order, int width, double* __restrict__ phi,
                            double* __restrict__ field) {
    td3_chain_wait();
    td3_chain_release();
    const i64 k = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= T.m) return;
    const i64 leaf = slot_leaf[k];
    if (leaf < 0) return;  // a slot left out (another rank's leaf)
    double lp, lx, ly;
    eval_local<LOCAL>(la, lb, leaf, order, width, T.pos[k] - T.center[2 * leaf],
                      T.pos[T.m + k] - T.center[2 * leaf + 1], lp, lx, ly);
    const i64 i = T.perm[k];
    if (POT) phi[i] += lp;
    field[i] += lx;
    field[T.m + i] += ly;
}

template <int LOCAL>
__global__ void k_far_adjoint(Targets T, Sources S, Adjoint A, const int* __restrict__ slot_leaf,
                              const double* __restrict__ fa, const double* __restrict__ fb,
                              const double* __restrict__ ba, const double* __restrict__ bb,
                              int order, int width) {
    td3_chain_wait();
    td3_chain_release();
    const i64 k = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= T.m) return;
    const i64 leaf = slot_leaf[k];
    if (leaf < 0) return;
    const double ux = T.pos[k] - T.center[2 * leaf], uy = T.pos[T.m + k] - T.center[2 * leaf + 1];
    const LocalJet f = local_jet<LOCAL>(fa, fb, leaf, order, width, ux, uy);  // Hessian
    const LocalJet b = local_jet<LOCAL>(ba, bb, leaf, order, width, ux, uy);  // Psi
    adjoint_far_add(f, b, k, T.perm[k], S.n, S, A);
}

// x in units of u relative to c, as an FP32 hi + lo pair.
__device__ __forceinline__ float2 split_rel(double x, double c, double inv_u) {
    const double v = (x - c) * inv_u;
    const float hi = (float)v;
    return make_float2(hi, (float)(v - (double)hi));
}

// Lanes (target, slice): targets t of the leaf in chunks of tsz, floor(32 / tsz) slices.
struct LaneMap {
    int tsz, slices, ti, slice;
    __device__ LaneMap(int count, int lane) {
        tsz = count < 32 ? count : 32;
        slices = 32 / tsz;
        ti = lane % tsz;
        slice = lane / tsz;
    }
    // v summed over the slices of each target into the slice-0 lane (fixed-order tree)
    template <int N>
    __device__ void sum_slices(double (&v)[N]) const {
        for (int off = 1; off < slices; off <<= 1) {
            const bool take = slice % (2 * off) == 0 && slice + off < slices;
#pragma unroll
            for (int c = 0; c < N; ++c) {
                const double o = __shfl_down_sync(0xffffffffu, v[c], off * tsz);
                if (take) v[c] += o;
            }
        }
    }
};

constexpr int NM_CAP = 128;  // staged sources per warp window (mixed forward)
// Warps per block of the mixed pair kernels: one, so a segment's warp frees its slot when
// it ends rather than with its block's slowest segment (segments differ in cost with
// their leaf's particles and partners); 32 one-warp blocks of 64 registers per SM.
constexpr int NM_WARPS = 1;

struct MixedWindow {
    float4 pos[NM_CAP];  // (x hi, x lo, y hi, y lo) relative to the target leaf's centre
    double q[NM_CAP];
    float qf[NM_CAP];
    int tag[NM_CAP];  // slot j (self-exclusion)
};

template <int KERNEL, bool POT, int NW>
__global__ void __launch_bounds__(32 * NW, 32 / NW)
k_near_mixed(Targets T, Sources S, i64 n_seg, const int* __restrict__ seg_leaf,
             const longlong2* __restrict__ seg_range, const i64* __restrict__ seg_out,
             const i64* __restrict__ partners, double eps2, double* __restrict__ partial,
             double* __restrict__ phi, double* __restrict__ field, i64* status) {
    td3_chain_wait();
    td3_chain_release();
    __shared__ MixedWindow windows[NW];
    const int lane = threadIdx.x & 31;
    MixedWindow& win = windows[threadIdx.x >> 5];
    const i64 seg = (i64)blockIdx.x * NW + (threadIdx.x >> 5);
    if (seg >= n_seg) return;
    const i64 leaf = seg_leaf[seg];
    const longlong2 er = seg_range[seg];
    const i64 outp = seg_out[seg];
    const i64 s0 = T.start[leaf];
    const int count = (int)(T.end[leaf] - s0);
    const LaneMap L(count, lane);
    const double u = pair_unit(S.unit), inv_u = 1.0 / u;
    const double cx = T.center[2 * leaf], cy = T.center[2 * leaf + 1];
    const float eps2f = (float)(eps2 * inv_u * inv_u);
    const i64 n = S.n;
    auto stage = [&](int p, i64 j) {
        const float2 x = split_rel(S.pos[j], cx, inv_u), y = split_rel(S.pos[n + j], cy, inv_u);
        win.pos[p] = make_float4(x.x, x.y, y.x, y.y);
        const double q = S.charge[j];
        win.q[p] = q;
        win.qf[p] = (float)q;
        win.tag[p] = (int)j;
    };
    for (int base = 0; base < count; base += L.tsz) {
        const int it = base + L.ti;
        const bool valid = L.slice < L.slices && it < count;
        const i64 k = s0 + (valid ? it : 0);
        const float2 X = split_rel(S.pos[k], cx, inv_u), Y = split_rel(S.pos[n + k], cy, inv_u);
        const bool qi_nonzero = S.charge[k] != 0.0;
        const int self = (int)k;
        KahanF kp, kx, ky;
        double qsum = 0.0;
        bool bad = false;
        for_source_windows<NM_CAP>(S, partners, er.x, er.y, lane, stage, [&](int wn) {
            if (!valid) return;
            const int step = L.slices;
            for (int p0 = L.slice; p0 < wn; p0 += NF_BLOCK * step) {
                float bp = 0.0f, bx = 0.0f, by = 0.0f;
                const int p1 = p0 + NF_BLOCK * step < wn ? p0 + NF_BLOCK * step : wn;
                for (int p = p0; p < p1; p += step) {
                    if (win.tag[p] == self) continue;
                    const float4 src = win.pos[p];
                    const float dx = (X.x - src.x) + (X.y - src.y);
                    const float dy = (Y.x - src.z) + (Y.y - src.w);
                    const float r2 = fmaf(dx, dx, fmaf(dy, dy, eps2f));
                    if (r2 == 0.0f) {  // coincident, unsoftened
                        bad |= qi_nonzero && win.q[p] != 0.0;
                        continue;
                    }
                    const float qj = win.qf[p];
                    if (KERNEL == TD3_KERNEL_LOG) {
                        if (POT) {
                            bp = fmaf(-qj, __logf(r2), bp);
                            qsum += win.q[p];
                        }
                        const float f = __fdividef(2.0f * qj, r2);
                        bx = fmaf(f, dx, bx);
                        by = fmaf(f, dy, by);
                    } else {
                        const float ir = rsqrtf(r2), qr = qj * ir, qr3 = qr * ir * ir;
                        bp += qr;
                        bx = fmaf(qr3, dx, bx);
                        by = fmaf(qr3, dy, by);
                    }
                }
                if (POT || KERNEL != TD3_KERNEL_LOG) kp.add(bp);
                kx.add(bx);
                ky.add(by);
            }
        });
        // back from units of u: log -ln u^2 sum q, 1/u; Coulomb 1/u, 1/u^2
        double v[3];
        if (KERNEL == TD3_KERNEL_LOG) {
            v[0] = kp.value() - 2.0 * log(u) * qsum;
            v[1] = kx.value() * inv_u;
            v[2] = ky.value() * inv_u;
        } else {
            v[0] = kp.value() * inv_u;
            v[1] = kx.value() * inv_u * inv_u;
            v[2] = ky.value() * inv_u * inv_u;
        }
        L.sum_slices(v);
        const unsigned badmask = __ballot_sync(0xffffffffu, bad && valid);
        if (valid && L.slice == 0) {
            if (outp < 0) {
                const i64 i = T.perm[k];
                phi[i] = POT ? v[0] : 0.0;
                field[i] = v[1];
                field[T.m + i] = v[2];
            } else {
                const i64 p = outp + it;
                partial[3 * p] = v[0];
                partial[3 * p + 1] = v[1];
                partial[3 * p + 2] = v[2];
            }
        }
        if (badmask && lane == __ffs(badmask) - 1) td3_report(status, T.perm[k] + 1);
    }
}

constexpr int NM_CAP_ADJ = 128;  // staged sources per warp window (mixed adjoint)

struct MixedAdjointWindow {
    float4 pos[NM_CAP_ADJ];  // as MixedWindow
    float4 qwe[NM_CAP_ADJ];  // (q, w, e_x / u, e_y / u)
    double w[NM_CAP_ADJ];    // the monopole in FP64 (its ln u^2 sum)
    int tag[NM_CAP_ADJ];
};

template <int KERNEL, int NW>
__global__ void __launch_bounds__(32 * NW, 32 / NW)
k_near_adjoint_mixed(Targets T, Sources S, Adjoint A, i64 n_seg, const int* __restrict__ seg_leaf,
                     const longlong2* __restrict__ seg_range, const i64* __restrict__ seg_out,
                     const i64* __restrict__ partners, double eps2, double* __restrict__ partial) {
    td3_chain_wait();
    td3_chain_release();
    __shared__ MixedAdjointWindow windows[NW];
    const int lane = threadIdx.x & 31;
    MixedAdjointWindow& win = windows[threadIdx.x >> 5];
    const i64 seg = (i64)blockIdx.x * NW + (threadIdx.x >> 5);
    if (seg >= n_seg) return;
    const i64 leaf = seg_leaf[seg];
    const longlong2 er = seg_range[seg];
    const i64 outp = seg_out[seg];
    const i64 s0 = T.start[leaf];
    const int count = (int)(T.end[leaf] - s0);
    const LaneMap L(count, lane);
    const i64 n = S.n;
    const double u = pair_unit(S.unit), inv_u = 1.0 / u;
    const double cx = T.center[2 * leaf], cy = T.center[2 * leaf + 1];
    const float eps2f = (float)(eps2 * inv_u * inv_u);
    auto stage = [&](int p, i64 j) {
        const float2 x = split_rel(S.pos[j], cx, inv_u), y = split_rel(S.pos[n + j], cy, inv_u);
        win.pos[p] = make_float4(x.x, x.y, y.x, y.y);
        const double w = A.weight[j];
        win.qwe[p] = make_float4((float)S.charge[j], (float)w, (float)(A.dipole[j] * inv_u),
                                 (float)(A.dipole[n + j] * inv_u));
        win.w[p] = w;
        win.tag[p] = (int)j;
    };
    for (int base = 0; base < count; base += L.tsz) {
        const int it = base + L.ti;
        const bool valid = L.slice < L.slices && it < count;
        const i64 k = s0 + (valid ? it : 0);
        const float2 X = split_rel(S.pos[k], cx, inv_u), Y = split_rel(S.pos[n + k], cy, inv_u);
        const int self = (int)k;
        KahanF kacc[6];
        double wsum = 0.0;
        for_source_windows<NM_CAP_ADJ>(S, partners, er.x, er.y, lane, stage, [&](int wn) {
            if (!valid) return;
            const int step = L.slices;
            for (int p0 = L.slice; p0 < wn; p0 += NF_BLOCK * step) {
                float blk[6] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
                const int p1 = p0 + NF_BLOCK * step < wn ? p0 + NF_BLOCK * step : wn;
                for (int p = p0; p < p1; p += step) {
                    if (win.tag[p] == self) continue;
                    const float4 src = win.pos[p];
                    const float dx = (X.x - src.x) + (X.y - src.y);
                    const float dy = (Y.x - src.z) + (Y.y - src.w);
                    if (eps2f == 0.0f && dx == 0.0f && dy == 0.0f) continue;  // coincident
                    const float4 c = win.qwe[p];
                    if (KERNEL == TD3_KERNEL_LOG) wsum += win.w[p];
                    adjoint_pair_mixed<KERNEL>(dx, dy, eps2f, c.x, c.y, c.z, c.w, blk);
                }
#pragma unroll
                for (int c = 0; c < 6; ++c) kacc[c].add(blk[c]);
            }
        });
        // back from units of u: the log kernel's sums scale as (1, 1/u, 1/u^2) plus
        // -ln u^2 sum w for Psi, the Coulomb kernel's as (1/u, 1/u^2, 1/u^3)
        const double sc = KERNEL == TD3_KERNEL_LOG ? 1.0 : inv_u;
        double acc[6];
        acc[0] = kacc[0].value() * sc;
        if (KERNEL == TD3_KERNEL_LOG) acc[0] -= 2.0 * log(u) * wsum;
        for (int c = 1; c < 3; ++c) acc[c] = kacc[c].value() * (sc * inv_u);
        for (int c = 3; c < 6; ++c) acc[c] = kacc[c].value() * (sc * inv_u * inv_u);
        L.sum_slices(acc);
        if (valid && L.slice == 0) {
            if (outp < 0) {
                adjoint_add(acc, k, T.perm[k], n, S, A);
            } else {
                const i64 p = outp + it;
                for (int c = 0; c < 6; ++c) partial[6 * p + c] = acc[c];
            }
        }
    }
}

struct NearArgs {
    Targets T;
    Sources S;
    i64 n_seg;
    const int* seg_leaf;
    const longlong2* seg_range;
    const i64* seg_out;
    const i64* partners;
    const double* la;
    const double* lb;
    int order, width;
    double eps2;
    double* partial;
    double* phi;
    double* field;
    i64* status;
};

template <int KERNEL, bool POT, bool OTHER, int LOCAL, bool MIXED>
int launch_near(const NearArgs& a, cudaStream_t s) {
    if (a.n_seg == 0) return TD3_OK;
    TD3_TRY(td3_launch_chained(k_near<KERNEL, POT, OTHER, LOCAL, MIXED>,
                               td3_blocks(a.n_seg, NW_NEAR), 32 * NW_NEAR, 0, s, a.T, a.S, a.n_seg, a.seg_leaf, a.seg_range, a.seg_out,
                               a.partners, a.la, a.lb, a.order, a.width, a.eps2, a.partial, a.phi,
                               a.field, a.status));
    TD3_TRY(td3_launch_chained(k_near_finish<POT, LOCAL>, td3_finish_blocks(a.n_seg), 32 * NF_WARPS, 0, s, a.T,
                               a.n_seg, a.seg_leaf, a.seg_out, a.la, a.lb, a.order, a.width,
                               a.partial, a.phi, a.field));
    TD3_CHECK_LAUNCH();
    return TD3_OK;
}

template <bool OTHER, int LOCAL>
int dispatch_near(int kernel, int with_potential, int mixed, const NearArgs& a, cudaStream_t s) {
    constexpr int LG = TD3_KERNEL_LOG, CL = TD3_KERNEL_COULOMB;
    if (kernel == LG) {
        if (with_potential)
            return mixed ? launch_near<LG, true, OTHER, LOCAL, true>(a, s)
                         : launch_near<LG, true, OTHER, LOCAL, false>(a, s);
        return mixed ? launch_near<LG, false, OTHER, LOCAL, true>(a, s)
                     : launch_near<LG, false, OTHER, LOCAL, false>(a, s);
    }
    if (with_potential)
        return mixed ? launch_near<CL, true, OTHER, LOCAL, true>(a, s)
                     : launch_near<CL, true, OTHER, LOCAL, false>(a, s);
    return mixed ? launch_near<CL, false, OTHER, LOCAL, true>(a, s)
                 : launch_near<CL, false, OTHER, LOCAL, false>(a, s);
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
    TD3_TRY(td3_launch_chained(k_plan_count, nb, 256, 0, s, n_nodes, rows, node_child, node_start,
                               node_end, segment, nseg, psize));
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
    TD3_TRY(td3_launch_chained(k_plan_fill, nb, 256, 0, s, n_nodes, rows, node_start, node_end,
                               segment, nseg_scan, psize_scan, nseg, seg_leaf,
                               reinterpret_cast<longlong2*>(seg_range), seg_out));
    TD3_CHECK_LAUNCH();
    return TD3_OK;
}

extern "C" int td3_fmm_evaluate(int kernel, const double* sorted_pos, const double* sorted_charge,
                                const int64_t* perm, int64_t n, const double* node_center,
                                const int64_t* node_start, const int64_t* node_end, int order,
                                const double* local_a, const double* local_b,
                                const int64_t* p2p_partners, const int* seg_leaf,
                                const int64_t* seg_range, const int64_t* seg_out, int64_t n_seg,
                                double* partial, double softening, int with_potential, int mixed,
                                double unit, double* phi, double* field, int64_t* status,
                                void* stream) {
    if (n < 0 || n_seg < 0 || order < 0 || order > TD3_MAX_ORDER) return TD3_EINVAL;
    if (mixed && !(unit > 0.0 && unit < INFINITY)) return TD3_EINVAL;
    if (kernel != TD3_KERNEL_COULOMB && kernel != TD3_KERNEL_LOG) return TD3_EINVAL;
    if (n == 0) return TD3_OK;
    bool lg = kernel == TD3_KERNEL_LOG;
    NearArgs a{Targets{sorted_pos, nullptr, perm, node_center, node_start, node_end, n},
               Sources{sorted_pos, sorted_charge, perm, node_start, node_end, n, unit},
               n_seg, seg_leaf, reinterpret_cast<const longlong2*>(seg_range), seg_out,
               p2p_partners, local_a, local_b, order,
               lg ? order + 1 : (order + 1) * (order + 2) / 2, softening * softening, partial,
               phi, field, status};
    cudaStream_t s = td3_stream(stream);
    if (lg) return dispatch_near<false, LOCAL_COMPLEX>(kernel, with_potential, mixed, a, s);
    return dispatch_near<false, LOCAL_CART>(kernel, with_potential, mixed, a, s);
}

template <int KERNEL, int LOCAL, bool MIXED>
int launch_adjoint(const Targets& T, const Sources& S, const Adjoint& A, i64 n_seg,
                   const int* seg_leaf, const longlong2* sr, const i64* seg_out,
                   const i64* partners, const double* fa, const double* fb, const double* ba,
                   const double* bb, int order, int width, double eps2, double* partial,
                   cudaStream_t s) {
    TD3_TRY(td3_launch_chained(k_near_adjoint<KERNEL, LOCAL, MIXED>, td3_blocks(n_seg, NW_NEAR),
                               32 * NW_NEAR, 0, s,
                               T, S, A, n_seg, seg_leaf, sr, seg_out, partners, fa, fb, ba, bb,
                               order, width, eps2, partial));
    TD3_TRY(td3_launch_chained(k_near_adjoint_finish<LOCAL>, td3_finish_blocks(n_seg), 32 * NF_WARPS, 0, s, T, S,
                               A, n_seg, seg_leaf, seg_out, fa, fb, ba, bb, order, width,
                               partial));
    return TD3_OK;
}

extern "C" int td3_fmm_adjoint(int kernel, const double* sorted_pos, const double* sorted_charge,
                               const int64_t* perm, int64_t n, const double* node_center,
                               const int64_t* node_start, const int64_t* node_end, int order,
                               const double* fwd_a, const double* fwd_b, const double* adj_a,
                               const double* adj_b, const int64_t* p2p_partners,
                               const int* seg_leaf, const int64_t* seg_range,
                               const int64_t* seg_out, int64_t n_seg, double* partial,
                               const double* sorted_weight, const double* sorted_dipole,
                               const double* efield, double softening, int mixed, double unit,
                               double* qbar, double* xbar, void* stream) {
    if (n < 0 || n_seg < 0 || order < 0 || order > TD3_MAX_ORDER) return TD3_EINVAL;
    if (mixed && !(unit > 0.0 && unit < INFINITY)) return TD3_EINVAL;
    if (kernel != TD3_KERNEL_COULOMB && kernel != TD3_KERNEL_LOG) return TD3_EINVAL;
    if (n == 0 || n_seg == 0) return TD3_OK;
    Targets T{sorted_pos, nullptr, perm, node_center, node_start, node_end, n};
    Sources S{sorted_pos, sorted_charge, perm, node_start, node_end, n, unit};
    Adjoint A{sorted_weight, sorted_dipole, efield, qbar, xbar};
    double eps2 = softening * softening;
    cudaStream_t s = td3_stream(stream);
    const longlong2* sr = reinterpret_cast<const longlong2*>(seg_range);
    if (kernel == TD3_KERNEL_LOG) {
        int width = order + 1;
        if (mixed)
            return launch_adjoint<TD3_KERNEL_LOG, LOCAL_COMPLEX, true>(
                T, S, A, n_seg, seg_leaf, sr, seg_out, p2p_partners, fwd_a, fwd_b, adj_a, adj_b,
                order, width, eps2, partial, s);
        return launch_adjoint<TD3_KERNEL_LOG, LOCAL_COMPLEX, false>(
            T, S, A, n_seg, seg_leaf, sr, seg_out, p2p_partners, fwd_a, fwd_b, adj_a, adj_b, order,
            width, eps2, partial, s);
    } else {
        int width = (order + 1) * (order + 2) / 2;
        if (mixed)
            return launch_adjoint<TD3_KERNEL_COULOMB, LOCAL_CART, true>(
                T, S, A, n_seg, seg_leaf, sr, seg_out, p2p_partners, fwd_a, fwd_b, adj_a, adj_b,
                order, width, eps2, partial, s);
        return launch_adjoint<TD3_KERNEL_COULOMB, LOCAL_CART, false>(
            T, S, A, n_seg, seg_leaf, sr, seg_out, p2p_partners, fwd_a, fwd_b, adj_a, adj_b, order,
            width, eps2, partial, s);
    }
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
                               int mixed, double unit, double* phi, double* field,
                               int64_t* status, void* stream) {
    if (m < 0 || n < 0 || n_seg < 0 || order < 0 || order > TD3_MAX_ORDER) return TD3_EINVAL;
    if (mixed && !(unit > 0.0 && unit < INFINITY)) return TD3_EINVAL;
    if (kernel != TD3_KERNEL_COULOMB && kernel != TD3_KERNEL_LOG) return TD3_EINVAL;
    if (m == 0) return TD3_OK;
    bool lg = kernel == TD3_KERNEL_LOG;
    NearArgs a{Targets{sorted_targets, sorted_exclude, target_perm, t_center, t_start, t_end, m},
               Sources{sorted_pos, sorted_charge, perm, s_start, s_end, n, unit},
               n_seg, seg_leaf, reinterpret_cast<const longlong2*>(seg_range), seg_out,
               p2p_partners, local_a, local_b, order,
               lg ? order + 1 : (order + 1) * (order + 2) / 2, softening * softening, partial,
               phi, field, status};
    cudaStream_t s = td3_stream(stream);
    if (lg) return dispatch_near<true, LOCAL_COMPLEX>(kernel, with_potential, mixed, a, s);
    return dispatch_near<true, LOCAL_CART>(kernel, with_potential, mixed, a, s);
}

extern "C" int td3_slot_leaves(int64_t n_nodes, const int64_t* node_child,
                               const int64_t* node_start, const int64_t* node_end,
                               int32_t* slot_leaf, void* stream) {
    if (n_nodes < 1 || n_nodes > 0x7fffffffLL) return TD3_EINVAL;
    TD3_TRY(td3_launch_chained(k_slot_leaves, td3_blocks(n_nodes, 256), 256, 0,
                               td3_stream(stream), n_nodes, node_child, node_start, node_end,
                               slot_leaf));
    TD3_CHECK_LAUNCH();
    return TD3_OK;
}

namespace {

constexpr int PART_NEAR = 1, PART_FAR = 2;

// The near part (pair sums written, then the multi-segment leaves) and / or the far part
// (local expansions added) of the mixed near field at the sources.
template <int KERNEL, bool POT, int LOCAL>
int launch_near_mixed(const NearArgs& a, const int* slot_leaf, int parts, cudaStream_t s) {
    if ((parts & PART_NEAR) && a.n_seg > 0) {
        TD3_TRY(td3_launch_chained(k_near_mixed<KERNEL, POT, NM_WARPS>,
                                   td3_blocks(a.n_seg, NM_WARPS), 32 * NM_WARPS, 0, s, a.T, a.S,
                                   a.n_seg, a.seg_leaf, a.seg_range, a.seg_out, a.partners,
                                   a.eps2, a.partial, a.phi, a.field, a.status));
        TD3_TRY(td3_launch_chained(k_near_finish<POT, LOCAL, true>, td3_finish_blocks(a.n_seg),
                                   32 * NF_WARPS, 0, s, a.T, a.n_seg, a.seg_leaf, a.seg_out, a.la,
                                   a.lb, a.order, a.width, a.partial, a.phi, a.field));
    }
    if (parts & PART_FAR)
        TD3_TRY(td3_launch_chained(k_far_field<LOCAL, POT>, td3_blocks(a.T.m, 256), 256, 0, s,
                                   a.T, slot_leaf, a.la, a.lb, a.order, a.width, a.phi, a.field));
    TD3_CHECK_LAUNCH();
    return TD3_OK;
}

template <int KERNEL, int LOCAL>
int launch_adjoint_mixed(const Targets& T, const Sources& S, const Adjoint& A,
                         const int* slot_leaf, i64 n_seg, const int* seg_leaf,
                         const longlong2* sr, const i64* seg_out, const i64* partners,
                         const double* fa, const double* fb, const double* ba, const double* bb,
                         int order, int width, double eps2, double* partial, int parts,
                         cudaStream_t s) {
    if ((parts & PART_NEAR) && n_seg > 0) {
        TD3_TRY(td3_launch_chained(k_near_adjoint_mixed<KERNEL, NM_WARPS>,
                                   td3_blocks(n_seg, NM_WARPS), 32 * NM_WARPS, 0, s, T, S, A,
                                   n_seg, seg_leaf, sr, seg_out, partners, eps2, partial));
        TD3_TRY(td3_launch_chained(k_near_adjoint_finish<LOCAL, true>, td3_finish_blocks(n_seg),
                                   32 * NF_WARPS, 0, s, T, S, A, n_seg, seg_leaf, seg_out, fa, fb,
                                   ba, bb, order, width, partial));
    }
    if (parts & PART_FAR)
        TD3_TRY(td3_launch_chained(k_far_adjoint<LOCAL>, td3_blocks(T.m, 256), 256, 0, s, T, S,
                                   A, slot_leaf, fa, fb, ba, bb, order, width));
    TD3_CHECK_LAUNCH();
    return TD3_OK;
}

int near_mixed(int kernel, const double* sorted_pos, const double* sorted_charge,
               const int64_t* perm, int64_t n, const double* node_center,
               const int64_t* node_start, const int64_t* node_end, int order,
               const double* local_a, const double* local_b, const int32_t* slot_leaf,
               const int64_t* p2p_partners, const int* seg_leaf, const int64_t* seg_range,
               const int64_t* seg_out, int64_t n_seg, double* partial, double softening,
               int with_potential, double unit, double* phi, double* field, int64_t* status,
               int parts, void* stream) {
    if (n < 0 || n_seg < 0 || order < 0 || order > TD3_MAX_ORDER) return TD3_EINVAL;
    if (!(unit > 0.0 && unit < INFINITY)) return TD3_EINVAL;
    if ((parts & PART_FAR) && !slot_leaf) return TD3_EINVAL;
    if (kernel != TD3_KERNEL_COULOMB && kernel != TD3_KERNEL_LOG) return TD3_EINVAL;
    if (n == 0) return TD3_OK;
    const bool lg = kernel == TD3_KERNEL_LOG;
    NearArgs a{Targets{sorted_pos, nullptr, perm, node_center, node_start, node_end, n},
               Sources{sorted_pos, sorted_charge, perm, node_start, node_end, n, unit},
               n_seg, seg_leaf, reinterpret_cast<const longlong2*>(seg_range), seg_out,
               p2p_partners, local_a, local_b, order,
               lg ? order + 1 : (order + 1) * (order + 2) / 2, softening * softening, partial,
               phi, field, status};
    cudaStream_t s = td3_stream(stream);
    constexpr int LG = TD3_KERNEL_LOG, CL = TD3_KERNEL_COULOMB;
    if (lg)
        return with_potential
                   ? launch_near_mixed<LG, true, LOCAL_COMPLEX>(a, slot_leaf, parts, s)
                   : launch_near_mixed<LG, false, LOCAL_COMPLEX>(a, slot_leaf, parts, s);
    return with_potential ? launch_near_mixed<CL, true, LOCAL_CART>(a, slot_leaf, parts, s)
                          : launch_near_mixed<CL, false, LOCAL_CART>(a, slot_leaf, parts, s);
}

int adjoint_mixed(int kernel, const double* sorted_pos, const double* sorted_charge,
                  const int64_t* perm, int64_t n, const double* node_center,
                  const int64_t* node_start, const int64_t* node_end, int order,
                  const double* fwd_a, const double* fwd_b, const double* adj_a,
                  const double* adj_b, const int32_t* slot_leaf, const int64_t* p2p_partners,
                  const int* seg_leaf, const int64_t* seg_range, const int64_t* seg_out,
                  int64_t n_seg, double* partial, const double* sorted_weight,
                  const double* sorted_dipole, const double* efield, double softening,
                  double unit, double* qbar, double* xbar, int parts, void* stream) {
    if (n < 0 || n_seg < 0 || order < 0 || order > TD3_MAX_ORDER) return TD3_EINVAL;
    if (!(unit > 0.0 && unit < INFINITY)) return TD3_EINVAL;
    if ((parts & PART_FAR) && !slot_leaf) return TD3_EINVAL;
    if (kernel != TD3_KERNEL_COULOMB && kernel != TD3_KERNEL_LOG) return TD3_EINVAL;
    if (n == 0) return TD3_OK;
    Targets T{sorted_pos, nullptr, perm, node_center, node_start, node_end, n};
    Sources S{sorted_pos, sorted_charge, perm, node_start, node_end, n, unit};
    Adjoint A{sorted_weight, sorted_dipole, efield, qbar, xbar};
    const double eps2 = softening * softening;
    cudaStream_t s = td3_stream(stream);
    const longlong2* sr = reinterpret_cast<const longlong2*>(seg_range);
    if (kernel == TD3_KERNEL_LOG)
        return launch_adjoint_mixed<TD3_KERNEL_LOG, LOCAL_COMPLEX>(
            T, S, A, slot_leaf, n_seg, seg_leaf, sr, seg_out, p2p_partners, fwd_a, fwd_b, adj_a,
            adj_b, order, order + 1, eps2, partial, parts, s);
    return launch_adjoint_mixed<TD3_KERNEL_COULOMB, LOCAL_CART>(
        T, S, A, slot_leaf, n_seg, seg_leaf, sr, seg_out, p2p_partners, fwd_a, fwd_b, adj_a, adj_b,
        order, (order + 1) * (order + 2) / 2, eps2, partial, parts, s);
}

}  // namespace

extern "C" int td3_fmm_evaluate_mixed(int kernel, const double* sorted_pos,
                                      const double* sorted_charge, const int64_t* perm, int64_t n,
                                      const double* node_center, const int64_t* node_start,
                                      const int64_t* node_end, int order, const double* local_a,
                                      const double* local_b, const int32_t* slot_leaf,
                                      const int64_t* p2p_partners, const int* seg_leaf,
                                      const int64_t* seg_range, const int64_t* seg_out,
                                      int64_t n_seg, double* partial, double softening,
                                      int with_potential, double unit, double* phi,
                                      double* field, int64_t* status, void* stream) {
    return near_mixed(kernel, sorted_pos, sorted_charge, perm, n, node_center, node_start,
                      node_end, order, local_a, local_b, slot_leaf, p2p_partners, seg_leaf,
                      seg_range, seg_out, n_seg, partial, softening, with_potential, unit, phi,
                      field, status, PART_NEAR | PART_FAR, stream);
}

extern "C" int td3_fmm_near_mixed(int kernel, const double* sorted_pos,
                                  const double* sorted_charge, const int64_t* perm, int64_t n,
                                  const double* node_center, const int64_t* node_start,
                                  const int64_t* node_end, const int64_t* p2p_partners,
                                  const int* seg_leaf, const int64_t* seg_range,
                                  const int64_t* seg_out, int64_t n_seg, double* partial,
                                  double softening, int with_potential, double unit, double* phi,
                                  double* field, int64_t* status, void* stream) {
    return near_mixed(kernel, sorted_pos, sorted_charge, perm, n, node_center, node_start,
                      node_end, 0, nullptr, nullptr, nullptr, p2p_partners, seg_leaf, seg_range,
                      seg_out, n_seg, partial, softening, with_potential, unit, phi, field,
                      status, PART_NEAR, stream);
}

extern "C" int td3_fmm_far_mixed(int kernel, const double* sorted_pos, const int64_t* perm,
                                 int64_t n, const double* node_center, int order,
                                 const double* local_a, const double* local_b,
                                 const int32_t* slot_leaf, int with_potential, double* phi,
                                 double* field, void* stream) {
    return near_mixed(kernel, sorted_pos, nullptr, perm, n, node_center, nullptr, nullptr, order,
                      local_a, local_b, slot_leaf, nullptr, nullptr, nullptr, nullptr, 0,
                      nullptr, 0.0, with_potential, 1.0, phi, field, nullptr, PART_FAR, stream);
}

extern "C" int td3_fmm_adjoint_mixed(int kernel, const double* sorted_pos,
                                     const double* sorted_charge, const int64_t* perm, int64_t n,
                                     const double* node_center, const int64_t* node_start,
                                     const int64_t* node_end, int order, const double* fwd_a,
                                     const double* fwd_b, const double* adj_a,
                                     const double* adj_b, const int32_t* slot_leaf,
                                     const int64_t* p2p_partners, const int* seg_leaf,
                                     const int64_t* seg_range, const int64_t* seg_out,
                                     int64_t n_seg, double* partial, const double* sorted_weight,
                                     const double* sorted_dipole, const double* efield,
                                     double softening, double unit, double* qbar, double* xbar,
                                     void* stream) {
    return adjoint_mixed(kernel, sorted_pos, sorted_charge, perm, n, node_center, node_start,
                         node_end, order, fwd_a, fwd_b, adj_a, adj_b, slot_leaf, p2p_partners,
                         seg_leaf, seg_range, seg_out, n_seg, partial, sorted_weight,
                         sorted_dipole, efield, softening, unit, qbar, xbar,
                         PART_NEAR | PART_FAR, stream);
}

extern "C" int td3_fmm_adjoint_near_mixed(int kernel, const double* sorted_pos,
                                          const double* sorted_charge, const int64_t* perm,
                                          int64_t n, const double* node_center,
                                          const int64_t* node_start, const int64_t* node_end,
                                          const int64_t* p2p_partners, const int* seg_leaf,
                                          const int64_t* seg_range, const int64_t* seg_out,
                                          int64_t n_seg, double* partial,
                                          const double* sorted_weight,
                                          const double* sorted_dipole, double softening,
                                          double unit, double* qbar, double* xbar, void* stream) {
    return adjoint_mixed(kernel, sorted_pos, sorted_charge, perm, n, node_center, node_start,
                         node_end, 0, nullptr, nullptr, nullptr, nullptr, nullptr, p2p_partners,
                         seg_leaf, seg_range, seg_out, n_seg, partial, sorted_weight,
                         sorted_dipole, nullptr, softening, unit, qbar, xbar, PART_NEAR, stream);
}

extern "C" int td3_fmm_adjoint_far_mixed(int kernel, const double* sorted_pos,
                                         const double* sorted_charge, const int64_t* perm,
                                         int64_t n, const double* node_center, int order,
                                         const double* fwd_a, const double* fwd_b,
                                         const double* adj_a, const double* adj_b,
                                         const int32_t* slot_leaf, const double* sorted_weight,
                                         const double* sorted_dipole, const double* efield,
                                         double* qbar, double* xbar, void* stream) {
    return adjoint_mixed(kernel, sorted_pos, sorted_charge, perm, n, node_center, nullptr,
                         nullptr, order, fwd_a, fwd_b, adj_a, adj_b, slot_leaf, nullptr, nullptr,
                         nullptr, nullptr, 0, nullptr, sorted_weight, sorted_dipole, efield, 0.0,
                         1.0, qbar, xbar, PART_FAR, stream);
}
