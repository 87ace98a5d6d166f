// The FMM of the softened Coulomb kernel in the plane with Cartesian expansions, FP64:
//   M2L by destination row  (K/cart_m2l_host/cart_m2l_host_pyccel.py:16-80)
//   L2L per level           (K/cart_downward/cart_downward_pyccel.py:14-55)
// (moments: moments.cu; L2P + P2P: nearfield.cu.)
//
// M2L: one warp per destination cell.  For each partner the warp builds the Taylor
// coefficients A_g(t), |g| <= p, of f = (|r|^2 + eps^2)^(-1/2) degree by degree in
// shared memory (the coefficients of one degree depend only on the two below), then
// every lane accumulates its local coefficients b over the M2L rows (b, a, a + b) of
// the reference's tables: T_b += coef * m_a * A_{a+b}.
#include "common.cuh"

namespace {

constexpr int CM2L_WARPS = 4;

__global__ void __launch_bounds__(32 * CM2L_WARPS)
k_m2l_cart(const i64* __restrict__ row_start, const i64* __restrict__ partners, i64 n_dst,
           const double* __restrict__ dst_center, const double* __restrict__ src_center,
           const double* __restrict__ moments, int order, double eps2,
           const int* __restrict__ row_a, const int* __restrict__ row_g,
           const double* __restrict__ row_coef, const int* __restrict__ b_start,
           double* __restrict__ local) {
    extern __shared__ double smem[];
    int n_coef = (order + 1) * (order + 2) / 2;
    int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    double* A = smem + (2 * wib) * n_coef;
    double* M = A + n_coef;
    constexpr int PER_LANE = 8;  // coefficients per lane held in registers
    for (i64 dst = (i64)blockIdx.x * CM2L_WARPS + wib; dst < n_dst; dst += (i64)gridDim.x * CM2L_WARPS) {
        i64 e0 = row_start[dst], e1 = row_start[dst + 1];
        if (e0 == e1) continue;
        double cx = dst_center[2 * dst], cy = dst_center[2 * dst + 1];
        for (int b0 = 0; b0 < n_coef; b0 += 32 * PER_LANE) {
            double acc[PER_LANE];
#pragma unroll
            for (int j = 0; j < PER_LANE; ++j) acc[j] = 0.0;
            for (i64 e = e0; e < e1; ++e) {
                i64 src = partners[e];
                double tx = cx - src_center[2 * src], ty = cy - src_center[2 * src + 1];
                double r2 = tx * tx + ty * ty + eps2;
                for (int i = lane; i < n_coef; i += 32) M[i] = moments[src * n_coef + i];
                if (lane == 0) A[0] = 1.0 / sqrt(r2);
                __syncwarp();
                for (int n = 1; n <= order; ++n) {
                    int base = n * (n + 1) / 2;
                    for (int b = lane; b <= n; b += 32) {
                        int a = n - b;
                        double s = 0.0;
                        if (a >= 1) s += (2 * n - 1) * tx * A[(n - 1) * n / 2 + b];
                        if (b >= 1) s += (2 * n - 1) * ty * A[(n - 1) * n / 2 + b - 1];
                        if (a >= 2) s += (n - 1) * A[(n - 2) * (n - 1) / 2 + b];
                        if (b >= 2) s += (n - 1) * A[(n - 2) * (n - 1) / 2 + b - 2];
                        A[base + b] = -s / (n * r2);
                    }
                    __syncwarp();
                }
#pragma unroll
                for (int j = 0; j < PER_LANE; ++j) {
                    int b = b0 + lane + 32 * j;
                    if (b < n_coef) {
                        double t = 0.0;
                        for (int r = b_start[b]; r < b_start[b + 1]; ++r)
                            t += row_coef[r] * M[row_a[r]] * A[row_g[r]];
                        acc[j] += t;
                    }
                }
                __syncwarp();
            }
#pragma unroll
            for (int j = 0; j < PER_LANE; ++j) {
                int b = b0 + lane + 32 * j;
                if (b < n_coef) local[dst * n_coef + b] += acc[j];
            }
        }
    }
}

// The same M2L for orders up to P (P = 4, 8, 12, 16) in scaled form and a lane per
// partner.  With m~_a = (-1)^|a| m_a / (a_x! a_y!) and A~_g = g_x! g_y! A_g, the rows
// (b, a, a + b) with coef = (-1)^|a| C(a_x + b_x, a_x) C(a_y + b_y, a_y) become
//   T_b = T~_b / (b_x! b_y!),  T~_b = sum_a m~_a A~_(a+b).
// A warp takes one destination and its partners CART_GROUP at a time: lane p < 8 builds
// partner p's A~ by the reference's recurrence (scaled, the last two degrees in
// registers) into a column of shared memory, lane 8 + p scales partner p's moments into
// another; then lane (q, p) = (lane / 8, lane % 8) forms partner p's share of T~_b for
// b = 4j + q, and three butterfly steps over p add the 8 shares (fixed order).
constexpr int CART_GROUP = 8;
constexpr int CART_LANE_MAX = 16;

constexpr int CART_CHUNK = 4;     // coefficients b of one degree per lane and pass
constexpr int CART_MAX_CHUNKS = 48;

struct CartScale {
    short bx[(CART_LANE_MAX + 1) * (CART_LANE_MAX + 2) / 2];
    short by[(CART_LANE_MAX + 1) * (CART_LANE_MAX + 2) / 2];
    double inv_fact2[(CART_LANE_MAX + 1) * (CART_LANE_MAX + 2) / 2];  // 1 / (a_x! a_y!)
    // runs of CART_CHUNK coefficients of one degree: degree nb, first b_y
    short chunk_nb[CART_MAX_CHUNKS], chunk_by[CART_MAX_CHUNKS];
    int n_chunks;
};

// Partner p's share of T~_b for the coefficients b = (nb - by, by), by = by0 ..
// by0 + CART_CHUNK - 1 (those with by <= nb): for each degree na of a the run of m~ (na +
// 1 values) and the run of A~ of degree na + nb from b_y = by0 on are read once, through
// a window of CART_CHUNK values of A~ that slides by one per a_y, so each value serves
// CART_CHUNK coefficients.  Each acc[r] sums over na, then a_y, in the order of the
// one-coefficient loop (the same bits).
template <typename T>
__device__ __forceinline__ void cart_chunk(const T* __restrict__ Mt, const T* __restrict__ At,
                                           int p, int nb, int by0, int order,
                                           T (&acc)[CART_CHUNK]) {
#pragma unroll
    for (int r = 0; r < CART_CHUNK; ++r) acc[r] = T(0);
    for (int na = 0; na + nb <= order; ++na) {
        int ng = na + nb, lim = ng - by0;  // the run of degree ng holds indices 0..lim
        const T* mrow = Mt + (na * (na + 1) / 2) * CART_GROUP + p;
        const T* grow = At + (ng * (ng + 1) / 2 + by0) * CART_GROUP + p;
        T w[CART_CHUNK];
#pragma unroll
        for (int r = 0; r < CART_CHUNK; ++r) w[r] = r <= lim ? grow[r * CART_GROUP] : T(0);
        for (int ay = 0; ay <= na; ++ay) {
            T m = mrow[ay * CART_GROUP];
#pragma unroll
            for (int r = 0; r < CART_CHUNK; ++r) acc[r] += m * w[r];
#pragma unroll
            for (int r = 0; r + 1 < CART_CHUNK; ++r) w[r] = w[r + 1];
            int k = ay + CART_CHUNK;
            w[CART_CHUNK - 1] = k <= lim ? grow[k * CART_GROUP] : T(0);
        }
    }
}

// The coefficient runs of cart_chunk for orders up to CART_LANE_MAX, degree by degree.
void cart_chunks(int order, CartScale& C) {
    C.n_chunks = 0;
    for (int nb = 0; nb <= order; ++nb)
        for (int by0 = 0; by0 <= nb; by0 += CART_CHUNK) {
            C.chunk_nb[C.n_chunks] = (short)nb;
            C.chunk_by[C.n_chunks] = (short)by0;
            ++C.n_chunks;
        }
}

template <int P>
__global__ void __launch_bounds__(32 * CM2L_WARPS)
k_m2l_cart_lanes(const i64* __restrict__ row_start, const i64* __restrict__ partners,
                 i64 n_dst, const double* __restrict__ dst_center,
                 const double* __restrict__ src_center, const double* __restrict__ moments,
                 int order, double eps2, const CartScale C, double* __restrict__ local) {
    constexpr int W = P + 1;
    extern __shared__ double cart_smem[];
    td3_chain_wait();
    td3_chain_release();
    int n_coef = (order + 1) * (order + 2) / 2;
    int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    int p = lane & (CART_GROUP - 1), q = lane >> 3;
    // per warp: A~ [g][partner], m~ [a][partner], T~ [b]; per block: the moments' scale
    // (-1)^|a| / (a_x! a_y!)
    double* At = cart_smem + (size_t)wib * (2 * CART_GROUP + 1) * n_coef;
    double* Mt = At + CART_GROUP * n_coef;
    double* T = Mt + CART_GROUP * n_coef;
    double* mscale = cart_smem + (size_t)CM2L_WARPS * (2 * CART_GROUP + 1) * n_coef;
    for (int a = threadIdx.x; a < n_coef; a += blockDim.x)
        mscale[a] = ((C.bx[a] + C.by[a]) & 1) ? -C.inv_fact2[a] : C.inv_fact2[a];
    __syncthreads();
    for (i64 dst = (i64)blockIdx.x * CM2L_WARPS + wib; dst < n_dst;
         dst += (i64)gridDim.x * CM2L_WARPS) {
        i64 e0 = row_start[dst], e1 = row_start[dst + 1];
        if (e0 == e1) continue;
        double cx = dst_center[2 * dst], cy = dst_center[2 * dst + 1];
        for (int b = lane; b < n_coef; b += 32) T[b] = 0.0;
        for (i64 base = e0; base < e1; base += CART_GROUP) {
            __syncwarp();
            bool live = base + p < e1;
            i64 src = live ? partners[base + p] : 0;
            if (lane < CART_GROUP) {
                double tx = cx - src_center[2 * src], ty = cy - src_center[2 * src + 1];
                // a lane past the row's end builds a zero column (finite scale)
                double r2 = live ? tx * tx + ty * ty + eps2 : 1.0;
                double prev2[W], prev1[W], cur[W];
                prev1[0] = live ? 1.0 / sqrt(r2) : 0.0;
                At[p] = prev1[0];
                double inv_r2 = 1.0 / r2;
#pragma unroll
                for (int n = 1; n < W; ++n) {
                    if (n > order) break;
                    double scale = -inv_r2 / n;
#pragma unroll
                    for (int gy = 0; gy <= n; ++gy) {
                        int gx = n - gy;
                        double s = 0.0;
                        if (gx >= 1) s += (2 * n - 1) * tx * gx * prev1[gy];
                        if (gy >= 1) s += (2 * n - 1) * ty * gy * prev1[gy - 1];
                        if (gx >= 2) s += (n - 1) * (gx * (gx - 1)) * prev2[gy];
                        if (gy >= 2) s += (n - 1) * (gy * (gy - 1)) * prev2[gy - 2];
                        cur[gy] = s * scale;
                        At[(n * (n + 1) / 2 + gy) * CART_GROUP + p] = cur[gy];
                    }
#pragma unroll
                    for (int k = 0; k < W; ++k) {
                        prev2[k] = prev1[k];
                        prev1[k] = cur[k];
                    }
                }
            }
            // the partners' scaled moments, every lane loading consecutive coefficients of
            // one partner at a time (coalesced, the loads of a partner in flight together)
            constexpr int NC = (P + 1) * (P + 2) / 2;
#pragma unroll 2
            for (int pp = 0; pp < CART_GROUP; ++pp) {
                const i64 s2 = __shfl_sync(0xffffffffu, src, pp);
                const bool l2 = __shfl_sync(0xffffffffu, live, pp);
                const double* m = moments + s2 * n_coef;
#pragma unroll
                for (int a0 = 0; a0 < NC; a0 += 32) {
                    const int a = a0 + lane;
                    if (a < n_coef) Mt[a * CART_GROUP + pp] = l2 ? m[a] * mscale[a] : 0.0;
                }
            }
            __syncwarp();
            // lane (q, p): chunks q, q + 4, ... of partner p, then 3 butterfly steps over p
            for (int k0 = 0; k0 < C.n_chunks; k0 += 4) {
                int k = k0 + q;
                int nb = k < C.n_chunks ? C.chunk_nb[k] : 0, by0 = k < C.n_chunks ? C.chunk_by[k] : 0;
                double acc[CART_CHUNK];
                if (k < C.n_chunks) {
                    cart_chunk<double>(Mt, At, p, nb, by0, order, acc);
                } else {
#pragma unroll
                    for (int r = 0; r < CART_CHUNK; ++r) acc[r] = 0.0;
                }
#pragma unroll
                for (int r = 0; r < CART_CHUNK; ++r) {
                    double a = acc[r];
                    a += __shfl_xor_sync(0xffffffffu, a, 4);
                    a += __shfl_xor_sync(0xffffffffu, a, 2);
                    a += __shfl_xor_sync(0xffffffffu, a, 1);
                    if (p == 0 && k < C.n_chunks && by0 + r <= nb)
                        T[nb * (nb + 1) / 2 + by0 + r] += a;
                }
            }
        }
        __syncwarp();
        for (int b = lane; b < n_coef; b += 32) local[dst * n_coef + b] += T[b] * C.inv_fact2[b];
    }
}

// The mixed-precision form of k_m2l_cart_lanes: the same partners-by-eight layout in
// FP32 on expansions scaled by a unit h = max(h_src, h_dst) per partner.  With t' = t / h,
// eps' = eps / h and m'_a = m_a / h^|a|, A_g(t; eps) = h^(-1-|g|) A_g(t'; eps'), so
// T_b = (1 / b!) h_d^(-1-|b|) sum_partners (h_d / h)^(1+|b|) S'_b with
// S'_b = sum_a m~'_a A~'_(a+b): every FP32 quantity O(1) and the factor at most 1 (a
// cell far smaller than its partner, which the lists hold, overflows neither way; inside
// one tree the factor is a power of two and exact), summed per destination in FP32 and
// added to the FP64 locals with the factor h_d^(-1-|b|) / b! in FP64.
template <int P>
__global__ void __launch_bounds__(32 * CM2L_WARPS)
k_m2l_cart_mixed(const i64* __restrict__ row_start, const i64* __restrict__ partners,
                 i64 n_dst, const double* __restrict__ dst_center,
                 const double* __restrict__ dst_half, const double* __restrict__ src_center,
                 const double* __restrict__ src_half, const double* __restrict__ moments,
                 int order, double eps2, const CartScale C, double* __restrict__ local) {
    constexpr int W = P + 1;
    extern __shared__ float cart_smem_f[];
    td3_chain_wait();
    td3_chain_release();
    int n_coef = (order + 1) * (order + 2) / 2;
    int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    int p = lane & (CART_GROUP - 1), q = lane >> 3;
    float* At = cart_smem_f + (size_t)wib * (2 * CART_GROUP + 1) * n_coef;
    float* Mt = At + CART_GROUP * n_coef;
    float* T = Mt + CART_GROUP * n_coef;
    // per block: the moments' scale (-1)^|a| / (a_x! a_y!) and degree |a|; per warp: the
    // partners' unit powers h^-n
    double* mscale = reinterpret_cast<double*>(
        cart_smem_f + (size_t)CM2L_WARPS * (2 * CART_GROUP + 1) * n_coef +
        ((CM2L_WARPS * (2 * CART_GROUP + 1) * n_coef) & 1));
    double* hpow = mscale + n_coef + (size_t)wib * CART_GROUP * (P + 1);
    int* mdeg = reinterpret_cast<int*>(mscale + n_coef + CM2L_WARPS * CART_GROUP * (P + 1));
    for (int a = threadIdx.x; a < n_coef; a += blockDim.x) {
        mscale[a] = ((C.bx[a] + C.by[a]) & 1) ? -C.inv_fact2[a] : C.inv_fact2[a];
        mdeg[a] = C.bx[a] + C.by[a];
    }
    __syncthreads();
    for (i64 dst = (i64)blockIdx.x * CM2L_WARPS + wib; dst < n_dst;
         dst += (i64)gridDim.x * CM2L_WARPS) {
        i64 e0 = row_start[dst], e1 = row_start[dst + 1];
        if (e0 == e1) continue;
        double cx = dst_center[2 * dst], cy = dst_center[2 * dst + 1], hd = dst_half[dst];
        for (int b = lane; b < n_coef; b += 32) T[b] = 0.0f;
        for (i64 base = e0; base < e1; base += CART_GROUP) {
            __syncwarp();
            bool live = base + p < e1;
            i64 src = live ? partners[base + p] : 0;
            // the partner's unit h = max(h_s, h_d): the moments / h^|a| and A~ at t / h stay
            // O(1), and (h_d / h)^(1 + |b|) <= 1 brings its sums to the destination's scale
            // (an exact power of two inside one tree)
            double hs = fmax(src_half[src], hd);
            const double ratio = hd / hs;
            if (lane < CART_GROUP) {
                double inv_h = 1.0 / hs;
                float tx = (float)((cx - src_center[2 * src]) * inv_h);
                float ty = (float)((cy - src_center[2 * src + 1]) * inv_h);
                float r2 = live ? (float)((double)tx * tx + (double)ty * ty + eps2 * inv_h * inv_h)
                                : 1.0f;
                float prev2[W], prev1[W], cur[W];
                prev1[0] = live ? rsqrtf(r2) : 0.0f;
                At[p] = prev1[0];
                float inv_r2 = 1.0f / r2;
#pragma unroll
                for (int n = 1; n < W; ++n) {
                    if (n > order) break;
                    float scale = -inv_r2 / n;
#pragma unroll
                    for (int gy = 0; gy <= n; ++gy) {
                        int gx = n - gy;
                        float s = 0.0f;
                        if (gx >= 1) s += (2 * n - 1) * tx * gx * prev1[gy];
                        if (gy >= 1) s += (2 * n - 1) * ty * gy * prev1[gy - 1];
                        if (gx >= 2) s += (n - 1) * (gx * (gx - 1)) * prev2[gy];
                        if (gy >= 2) s += (n - 1) * (gy * (gy - 1)) * prev2[gy - 2];
                        cur[gy] = s * scale;
                        At[(n * (n + 1) / 2 + gy) * CART_GROUP + p] = cur[gy];
                    }
#pragma unroll
                    for (int k = 0; k < W; ++k) {
                        prev2[k] = prev1[k];
                        prev1[k] = cur[k];
                    }
                }
            } else if (lane < 2 * CART_GROUP) {
                // partner p's powers h^-n, n <= order
                double inv_h = 1.0 / hs, pw = 1.0;
                for (int n = 0; n <= order; ++n, pw *= inv_h) hpow[p * (P + 1) + n] = pw;
            }
            __syncwarp();
            // the partners' moments in units of their h, every lane loading consecutive
            // coefficients of one partner at a time (coalesced, the loads of a partner in
            // flight together)
            constexpr int NC = (P + 1) * (P + 2) / 2;
#pragma unroll 2
            for (int pp = 0; pp < CART_GROUP; ++pp) {
                const i64 s2 = __shfl_sync(0xffffffffu, src, pp);
                const bool l2 = __shfl_sync(0xffffffffu, live, pp);
                const double* m = moments + s2 * n_coef;
#pragma unroll
                for (int a0 = 0; a0 < NC; a0 += 32) {
                    const int a = a0 + lane;
                    if (a < n_coef)
                        Mt[a * CART_GROUP + pp] =
                            l2 ? (float)(m[a] * mscale[a] * hpow[pp * (P + 1) + mdeg[a]]) : 0.0f;
                }
            }
            // ratio^(1 + nb) for this lane's chunks (their degrees only grow)
            double rpow = ratio;
            int rpow_nb = 0;
            __syncwarp();
            for (int k0 = 0; k0 < C.n_chunks; k0 += 4) {
                int k = k0 + q;
                int nb = k < C.n_chunks ? C.chunk_nb[k] : 0, by0 = k < C.n_chunks ? C.chunk_by[k] : 0;
                float acc[CART_CHUNK];
                for (; rpow_nb < nb; ++rpow_nb) rpow *= ratio;
                const float sc = (float)rpow;
                if (k < C.n_chunks) {
                    cart_chunk<float>(Mt, At, p, nb, by0, order, acc);
                } else {
#pragma unroll
                    for (int r = 0; r < CART_CHUNK; ++r) acc[r] = 0.0f;
                }
#pragma unroll
                for (int r = 0; r < CART_CHUNK; ++r) {
                    float a = acc[r] * sc;
                    a += __shfl_xor_sync(0xffffffffu, a, 4);
                    a += __shfl_xor_sync(0xffffffffu, a, 2);
                    a += __shfl_xor_sync(0xffffffffu, a, 1);
                    if (p == 0 && k < C.n_chunks && by0 + r <= nb)
                        T[nb * (nb + 1) / 2 + by0 + r] += a;
                }
            }
        }
        __syncwarp();
        double inv_hd = 1.0 / hd;
        for (int b = lane; b < n_coef; b += 32) {
            int nb = C.bx[b] + C.by[b];
            double scale = inv_hd;
            for (int k = 0; k < nb; ++k) scale *= inv_hd;
            local[dst * n_coef + b] += (double)T[b] * C.inv_fact2[b] * scale;
        }
    }
}

CartScale cart_scale(int order) {
    CartScale C{};
    double f[CART_LANE_MAX + 1];
    f[0] = 1.0;
    for (int k = 1; k <= CART_LANE_MAX; ++k) f[k] = f[k - 1] * k;
    for (int n = 0; n <= order; ++n)
        for (int y = 0; y <= n; ++y) {
            int i = n * (n + 1) / 2 + y;
            C.bx[i] = (short)(n - y);
            C.by[i] = (short)y;
            C.inv_fact2[i] = 1.0 / (f[n - y] * f[y]);
        }
    cart_chunks(order, C);
    return C;
}

// L2L of one level: a block per (node, child), thread b: T_b(child) += sum_g C(g, b) T_g
// s^(g-b) over the rows of b (g, d = g - b, coef).  The monomials s^d are built once per
// block into shared memory, column d_y by thread d_y as the reference's mono recurrence
// builds them (d_y factors of s_y, then s_x one at a time).
__global__ void k_l2l_cart(i64 lo, int order, int n_coef, const double* __restrict__ center,
                           const i64* __restrict__ child, const int* __restrict__ l2l_start,
                           const int* __restrict__ l2l_g, const int* __restrict__ l2l_d,
                           const double* __restrict__ l2l_coef, double* __restrict__ local) {
    extern __shared__ double shift_mono[];
    i64 node = lo + blockIdx.x / 4;
    i64 first = child[node];
    if (first < 0) return;  // the whole block: a leaf has no children
    i64 ch = first + (blockIdx.x & 3);
    double sx = center[2 * ch] - center[2 * node], sy = center[2 * ch + 1] - center[2 * node + 1];
    for (int dy = threadIdx.x; dy <= order; dy += blockDim.x) {
        double mono = 1.0;
        for (int k = 0; k < dy; ++k) mono = mono * sy;
        for (int dx = 0; dx + dy <= order; ++dx) {
            shift_mono[(dx + dy) * (dx + dy + 1) / 2 + dy] = mono;
            mono = mono * sx;
        }
    }
    __syncthreads();
    for (int b = threadIdx.x; b < n_coef; b += blockDim.x) {
        double acc = 0.0;
        for (int r = l2l_start[b]; r < l2l_start[b + 1]; ++r)
            acc += l2l_coef[r] * local[node * n_coef + l2l_g[r]] * shift_mono[l2l_d[r]];
        local[ch * n_coef + b] += acc;
    }
}

}  // namespace

extern "C" int td3_cart_m2l(const int64_t* row_start, const int64_t* partners, int64_t n_dst,
                            const double* dst_center, const double* src_center,
                            const double* moments, int order, double softening,
                            const int* row_a, const int* row_g, const double* row_coef,
                            const int* b_start, double* local, void* stream) {
    if (n_dst < 0 || order < 0 || order > TD3_MAX_ORDER) return TD3_EINVAL;
    if (n_dst == 0) return TD3_OK;
    cudaStream_t s = td3_stream(stream);
    int n_coef = (order + 1) * (order + 2) / 2;
    if (order <= CART_LANE_MAX) {
        CartScale C{};
        double f[CART_LANE_MAX + 1];
        f[0] = 1.0;
        for (int k = 1; k <= CART_LANE_MAX; ++k) f[k] = f[k - 1] * k;
        for (int n = 0; n <= order; ++n)
            for (int y = 0; y <= n; ++y) {
                int i = n * (n + 1) / 2 + y;
                C.bx[i] = (short)(n - y);
                C.by[i] = (short)y;
                C.inv_fact2[i] = 1.0 / (f[n - y] * f[y]);
            }
        cart_chunks(order, C);
        size_t lane_smem = sizeof(double) * ((2 * CART_GROUP + 1) * n_coef * CM2L_WARPS + n_coef);
        i64 nb = (n_dst + CM2L_WARPS - 1) / CM2L_WARPS;
        unsigned grid = (unsigned)(nb < 148 * 64 ? nb : 148 * 64);
        auto run = [&](auto kernel) -> int {
            TD3_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)lane_smem));
            TD3_TRY(td3_launch_chained(kernel, grid, 32 * CM2L_WARPS, lane_smem, s, row_start,
                                       partners, n_dst, dst_center, src_center, moments, order,
                                       softening * softening, C, local));
            return TD3_OK;
        };
        if (order <= 4) return run(k_m2l_cart_lanes<4>);
        if (order <= 8) return run(k_m2l_cart_lanes<8>);
        if (order <= 12) return run(k_m2l_cart_lanes<12>);
        return run(k_m2l_cart_lanes<16>);
    }
    size_t smem = sizeof(double) * 2 * n_coef * CM2L_WARPS;
    if (smem > 48 * 1024)
        TD3_TRY(cudaFuncSetAttribute(k_m2l_cart, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem));
    i64 blocks = (n_dst + CM2L_WARPS - 1) / CM2L_WARPS;
    if (blocks > 148 * 64) blocks = 148 * 64;
    k_m2l_cart<<<(unsigned)blocks, 32 * CM2L_WARPS, smem, s>>>(
        row_start, partners, n_dst, dst_center, src_center, moments, order,
        softening * softening, row_a, row_g, row_coef, b_start, local);
    TD3_CHECK_LAUNCH();
    return TD3_OK;
}

extern "C" int td3_cart_downward(const int64_t* levels, int64_t n_levels, const double* node_center,
                                 const int64_t* node_child, int order, const int64_t* ex,
                                 const int64_t* ey, const int* l2l_start, const int* l2l_g,
                                 const int* l2l_d, const double* l2l_coef, double* local,
                                 void* stream) {
    if (n_levels < 1 || order < 0 || order > TD3_MAX_ORDER) return TD3_EINVAL;
    cudaStream_t s = td3_stream(stream);
    int n_coef = (order + 1) * (order + 2) / 2;
    unsigned threads = (unsigned)((n_coef + 31) / 32 * 32);
    if (threads > 256) threads = 256;
    size_t smem = sizeof(double) * n_coef;
    if (smem > 48 * 1024)
        TD3_TRY(cudaFuncSetAttribute(k_l2l_cart, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem));
    (void)ex;
    (void)ey;
    for (i64 level = 0; level + 1 < n_levels; ++level) {
        i64 lo = levels[level], hi = levels[level + 1];
        if (hi <= lo) continue;
        k_l2l_cart<<<(unsigned)(4 * (hi - lo)), threads, smem, s>>>(
            lo, order, n_coef, node_center, node_child, l2l_start, l2l_g, l2l_d, l2l_coef, local);
    }
    TD3_CHECK_LAUNCH();
    return TD3_OK;
}

extern "C" int td3_cart_m2l_mixed(const int64_t* row_start, const int64_t* partners,
                                  int64_t n_dst, const double* dst_center,
                                  const double* dst_half, const double* src_center,
                                  const double* src_half, const double* moments, int order,
                                  double softening, double* local, void* stream) {
    if (n_dst < 0 || order < 0 || order > CART_LANE_MAX) return TD3_EINVAL;
    if (n_dst == 0) return TD3_OK;
    cudaStream_t s = td3_stream(stream);
    int n_coef = (order + 1) * (order + 2) / 2;
    CartScale C = cart_scale(order);
    // per-warp areas (floats, padded to 8 bytes), the scale table, the unit powers, degrees
    size_t smem = sizeof(float) * ((2 * CART_GROUP + 1) * n_coef * CM2L_WARPS + 1) +
                  sizeof(double) * (n_coef + CM2L_WARPS * CART_GROUP * (CART_LANE_MAX + 1)) +
                  sizeof(int) * n_coef;
    i64 nb = (n_dst + CM2L_WARPS - 1) / CM2L_WARPS;
    unsigned grid = (unsigned)(nb < 148 * 64 ? nb : 148 * 64);
    auto run = [&](auto kernel) -> int {
        TD3_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem));
        TD3_TRY(td3_launch_chained(kernel, grid, 32 * CM2L_WARPS, smem, s, row_start, partners,
                                   n_dst, dst_center, dst_half, src_center, src_half, moments,
                                   order, softening * softening, C, local));
        return TD3_OK;
    };
    if (order <= 4) return run(k_m2l_cart_mixed<4>);
    if (order <= 8) return run(k_m2l_cart_mixed<8>);
    if (order <= 12) return run(k_m2l_cart_mixed<12>);
    return run(k_m2l_cart_mixed<16>);
}
