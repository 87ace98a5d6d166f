// Cell moments, leaves from their particles and parents by M2M, deepest level first:
//   Coulomb  Q, sum|q|, p, S (K/quadtree_moments_upward/quadtree_moments_upward_pyccel.py:13-83)
//   log      a_n = sum q (z - c)^n   (K/log_moments_upward/log_moments_upward_pyccel.py:14-93)
//   Cartesian m_g = sum q (r - c)^g  (K/cart_moments_upward/cart_moments_upward_pyccel.py:14-82)
// The particles are read in tree order (sorted positions and charges, contiguous per
// leaf).  Each output coefficient is summed by one thread in the reference's order,
// and this file is compiled with --fmad=false, so the moments equal the reference's
// bit for bit.
#include "common.cuh"

namespace {

constexpr int MOM_THREADS = 128;

__global__ void k_coulomb_moments(i64 lo, i64 hi, const double* __restrict__ spos,
                                  const double* __restrict__ scharge, i64 n,
                                  const double* __restrict__ node_center,
                                  const i64* __restrict__ node_start,
                                  const i64* __restrict__ node_end,
                                  const i64* __restrict__ node_child, double* node_q,
                                  double* node_qabs, double* node_p, double* node_s) {
    i64 node = lo + (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (node >= hi) return;
    double q = 0.0, qabs = 0.0, px = 0.0, py = 0.0, sxx = 0.0, sxy = 0.0, syy = 0.0;
    double xmid = node_center[2 * node], ymid = node_center[2 * node + 1];
    i64 first = node_child[node];
    if (first < 0) {
        for (i64 k = node_start[node]; k < node_end[node]; ++k) {
            double c = scharge[k];
            double dx = spos[k] - xmid;
            double dy = spos[n + k] - ymid;
            q += c;
            qabs += fabs(c);
            px += c * dx;
            py += c * dy;
            sxx += c * dx * dx;
            sxy += c * dx * dy;
            syy += c * dy * dy;
        }
    } else {
        for (i64 child = first; child < first + 4; ++child) {
            double dx = node_center[2 * child] - xmid;
            double dy = node_center[2 * child + 1] - ymid;
            double cq = node_q[child], cpx = node_p[2 * child], cpy = node_p[2 * child + 1];
            q += cq;
            qabs += node_qabs[child];
            px += cpx + cq * dx;
            py += cpy + cq * dy;
            sxx += node_s[3 * child] + 2.0 * cpx * dx + cq * dx * dx;
            sxy += node_s[3 * child + 1] + cpx * dy + cpy * dx + cq * dx * dy;
            syy += node_s[3 * child + 2] + 2.0 * cpy * dy + cq * dy * dy;
        }
    }
    node_q[node] = q;
    node_qabs[node] = qabs;
    node_p[2 * node] = px;
    node_p[2 * node + 1] = py;
    node_s[3 * node] = sxx;
    node_s[3 * node + 1] = sxy;
    node_s[3 * node + 2] = syy;
}

// One thread per (node, n), n = 0..order.  sdip (2, n_particles; may be null) adds
// point dipoles e = (ex, ey) at the particles: a_n -= n e (z - c)^(n - 1), the moments
// of the adjoint (transposed) FMM pass, whose sources are monopoles and dipoles.
__global__ void k_log_moments(i64 lo, i64 hi, int order, const double* __restrict__ spos,
                              const double* __restrict__ scharge, i64 n_particles,
                              const double* __restrict__ node_center,
                              const i64* __restrict__ node_start, const i64* __restrict__ node_end,
                              const i64* __restrict__ node_child,
                              const double* __restrict__ binomial, int bsize, double* node_qabs,
                              double* moment_re, double* moment_im,
                              const double* __restrict__ sdip) {
    i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    int w = order + 1;
    i64 node = lo + t / w;
    int n = (int)(t % w);
    if (node >= hi) return;
    double xmid = node_center[2 * node], ymid = node_center[2 * node + 1];
    double acc_re = 0.0, acc_im = 0.0, qabs = 0.0;
    i64 first = node_child[node];
    if (first < 0) {
        for (i64 k = node_start[node]; k < node_end[node]; ++k) {
            double q = scharge[k];
            qabs += fabs(q);
            double dx = spos[k] - xmid, dy = spos[n_particles + k] - ymid;
            double pr = q, pi = 0.0;
            for (int m = 0; m < n; ++m) {
                double next_re = pr * dx - pi * dy;
                pi = pr * dy + pi * dx;
                pr = next_re;
            }
            acc_re += pr;
            acc_im += pi;
            if (sdip && n > 0) {
                // - n e (z - c)^(n-1)
                double er = sdip[k], ei = sdip[n_particles + k];
                double zr = 1.0, zi = 0.0;
                for (int m = 0; m < n - 1; ++m) {
                    double nr = zr * dx - zi * dy;
                    zi = zr * dy + zi * dx;
                    zr = nr;
                }
                acc_re -= n * (er * zr - ei * zi);
                acc_im -= n * (er * zi + ei * zr);
            }
        }
    } else {
        double sh_re[TD3_MAX_ORDER + 1], sh_im[TD3_MAX_ORDER + 1];
        for (i64 child = first; child < first + 4; ++child) {
            qabs += node_qabs[child];
            if (node_end[child] == node_start[child]) continue;
            double s_re = node_center[2 * child] - xmid;
            double s_im = node_center[2 * child + 1] - ymid;
            sh_re[0] = 1.0;
            sh_im[0] = 0.0;
            for (int k = 1; k <= n; ++k) {
                sh_re[k] = sh_re[k - 1] * s_re - sh_im[k - 1] * s_im;
                sh_im[k] = sh_re[k - 1] * s_im + sh_im[k - 1] * s_re;
            }
            double c_re = 0.0, c_im = 0.0;
            for (int m = 0; m <= n; ++m) {
                double c = binomial[n * bsize + m];
                double a_re = moment_re[child * w + m] * c;
                double a_im = moment_im[child * w + m] * c;
                c_re += a_re * sh_re[n - m] - a_im * sh_im[n - m];
                c_im += a_re * sh_im[n - m] + a_im * sh_re[n - m];
            }
            acc_re += c_re;
            acc_im += c_im;
        }
    }
    moment_re[node * w + n] = acc_re;
    moment_im[node * w + n] = acc_im;
    if (n == 0) node_qabs[node] = qabs;
}


// The leaf moments with one thread per leaf and every coefficient in registers (orders
// up to P, compile-time loop bounds), every leaf of the tree in one launch; the
// operations and their order per coefficient are those of k_log_moments, so the
// results are the same bits.
template <int P>
__global__ void k_log_leaf_moments(i64 count, int order, const double* __restrict__ spos,
                                   const double* __restrict__ scharge, i64 n_particles,
                                   const double* __restrict__ node_center,
                                   const i64* __restrict__ node_start,
                                   const i64* __restrict__ node_end,
                                   const i64* __restrict__ node_child, double* node_qabs,
                                   double* moment_re, double* moment_im,
                                   const double* __restrict__ sdip) {
    td3_chain_wait();
    td3_chain_release();
    constexpr int W = P + 1;
    i64 node = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (node >= count || node_child[node] >= 0) return;
    int w = order + 1;
    double xmid = node_center[2 * node], ymid = node_center[2 * node + 1];
    double ar[W], ai[W];
#pragma unroll
    for (int n = 0; n < W; ++n) ar[n] = ai[n] = 0.0;
    double qabs = 0.0;
    for (i64 k = node_start[node]; k < node_end[node]; ++k) {
        double q = scharge[k];
        qabs += fabs(q);
        double dx = spos[k] - xmid, dy = spos[n_particles + k] - ymid;
        double pr = q, pi = 0.0;
#pragma unroll
        for (int n = 0; n < W; ++n) {
            ar[n] += pr;
            ai[n] += pi;
            double next_re = pr * dx - pi * dy;
            pi = pr * dy + pi * dx;
            pr = next_re;
        }
        if (sdip) {
            double er = sdip[k], ei = sdip[n_particles + k];
            double zr = 1.0, zi = 0.0;
#pragma unroll
            for (int n = 1; n < W; ++n) {
                ar[n] -= n * (er * zr - ei * zi);
                ai[n] -= n * (er * zi + ei * zr);
                double nr = zr * dx - zi * dy;
                zi = zr * dy + zi * dx;
                zr = nr;
            }
        }
    }
#pragma unroll
    for (int n = 0; n < W; ++n) {
        if (n < w) {
            moment_re[node * w + n] = ar[n];
            moment_im[node * w + n] = ai[n];
        }
    }
    node_qabs[node] = qabs;
}

// M2M of the internal nodes of one level, a thread per (node, child) with the child's
// coefficients and the powers of its shift in registers (orders up to P): each thread
// forms its child's shifted coefficients c_n = sum_m C(n, m) a_m s^(n-m) in the order of
// k_log_moments into shared memory, then a thread per (node, n) adds the four children
// in order.  The operations are those of k_log_moments, so the results are the same bits.
constexpr int M2M_NODES = 32;  // nodes per block (4 threads each)

template <int P>
__global__ void __launch_bounds__(M2M_NODES * 4)
k_log_m2m_level(i64 lo, i64 hi, int order, const double* __restrict__ node_center,
                const i64* __restrict__ node_start, const i64* __restrict__ node_end,
                const i64* __restrict__ node_child, const double* __restrict__ binomial,
                int bsize, double* node_qabs, double* moment_re, double* moment_im) {
    constexpr int W = P + 1;
    __shared__ double2 shifted[M2M_NODES][4][W];
    __shared__ int present[M2M_NODES][4];
    td3_chain_wait();
    td3_chain_release();
    int w = order + 1;
    int local = threadIdx.x >> 2, c = threadIdx.x & 3;
    i64 node = lo + (i64)blockIdx.x * M2M_NODES + local;
    int has = 0;
    if (node < hi) {
        i64 first = node_child[node];
        if (first >= 0) {
            i64 child = first + c;
            has = node_end[child] != node_start[child];
            if (has) {
                double s_re = node_center[2 * child] - node_center[2 * node];
                double s_im = node_center[2 * child + 1] - node_center[2 * node + 1];
                double sh_re[W], sh_im[W], cr[W], ci[W];
                sh_re[0] = 1.0;
                sh_im[0] = 0.0;
#pragma unroll
                for (int n = 1; n < W; ++n) {
                    sh_re[n] = sh_re[n - 1] * s_re - sh_im[n - 1] * s_im;
                    sh_im[n] = sh_re[n - 1] * s_im + sh_im[n - 1] * s_re;
                }
#pragma unroll
                for (int m = 0; m < W; ++m) {
                    cr[m] = m < w ? moment_re[child * w + m] : 0.0;
                    ci[m] = m < w ? moment_im[child * w + m] : 0.0;
                }
#pragma unroll
                for (int n = 0; n < W; ++n) {
                    double c_re = 0.0, c_im = 0.0;
#pragma unroll
                    for (int m = 0; m <= n; ++m) {
                        double b = binomial[n * bsize + m];
                        double a_re = cr[m] * b, a_im = ci[m] * b;
                        c_re += a_re * sh_re[n - m] - a_im * sh_im[n - m];
                        c_im += a_re * sh_im[n - m] + a_im * sh_re[n - m];
                    }
                    shifted[local][c][n] = make_double2(c_re, c_im);
                }
            }
        } else {
            has = -1;  // a leaf: its moments come from its particles
        }
    } else {
        has = -1;
    }
    present[local][c] = has;
    __syncthreads();
    for (int item = threadIdx.x; item < M2M_NODES * w; item += blockDim.x) {
        int k = item / w, n = item - k * w;
        i64 out = lo + (i64)blockIdx.x * M2M_NODES + k;
        if (present[k][0] < 0) continue;
        double acc_re = 0.0, acc_im = 0.0;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            if (!present[k][j]) continue;
            double2 v = shifted[k][j][n];
            acc_re += v.x;
            acc_im += v.y;
        }
        moment_re[out * w + n] = acc_re;
        moment_im[out * w + n] = acc_im;
        if (n == 0) {
            i64 first = node_child[out];
            double qabs = 0.0;
            for (i64 child = first; child < first + 4; ++child) qabs += node_qabs[child];
            node_qabs[out] = qabs;
        }
    }
}

// The whole upward pass in one launch (orders up to P): a thread per node.  A leaf's
// thread forms its moments from its particles with the operations of
// k_log_leaf_moments, then arrives at its parent; the fourth child to arrive forms the
// parent by M2M with the operations of k_log_m2m_level (each child's shifted
// coefficients c_n = sum_m C(n, m) a_m s^(n-m), the children added in order) and goes on
// up.  The moments are therefore the same bits as the level-by-level pass.  No thread
// waits for another: the last arrival does the work, a fence before each arrival
// publishes the arriving node's moments, and the children are read through L2.
template <int P>
__global__ void __launch_bounds__(MOM_THREADS)
k_log_moments_tree(i64 count, int order, const double* __restrict__ spos,
                   const double* __restrict__ scharge, i64 n_particles,
                   const double* __restrict__ node_center, const i64* __restrict__ node_start,
                   const i64* __restrict__ node_end, const i64* __restrict__ node_child,
                   const int* __restrict__ parent, const double* __restrict__ binomial,
                   int bsize, double* node_qabs, double* moment_re, double* moment_im,
                   const double* __restrict__ sdip, int* arrive) {
    constexpr int W = P + 1;
    i64 node = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (node >= count || node_child[node] >= 0) return;
    const int w = order + 1;
    {
        double xmid = node_center[2 * node], ymid = node_center[2 * node + 1];
        double ar[W], ai[W];
#pragma unroll
        for (int n = 0; n < W; ++n) ar[n] = ai[n] = 0.0;
        double qabs = 0.0;
        for (i64 k = node_start[node]; k < node_end[node]; ++k) {
            double q = scharge[k];
            qabs += fabs(q);
            double dx = spos[k] - xmid, dy = spos[n_particles + k] - ymid;
            double pr = q, pi = 0.0;
#pragma unroll
            for (int n = 0; n < W; ++n) {
                ar[n] += pr;
                ai[n] += pi;
                double next_re = pr * dx - pi * dy;
                pi = pr * dy + pi * dx;
                pr = next_re;
            }
            if (sdip) {
                double er = sdip[k], ei = sdip[n_particles + k];
                double zr = 1.0, zi = 0.0;
#pragma unroll
                for (int n = 1; n < W; ++n) {
                    ar[n] -= n * (er * zr - ei * zi);
                    ai[n] -= n * (er * zi + ei * zr);
                    double nr = zr * dx - zi * dy;
                    zi = zr * dy + zi * dx;
                    zr = nr;
                }
            }
        }
#pragma unroll
        for (int n = 0; n < W; ++n) {
            if (n < w) {
                moment_re[node * w + n] = ar[n];
                moment_im[node * w + n] = ai[n];
            }
        }
        node_qabs[node] = qabs;
    }
    for (i64 cur = node;;) {
        int up = parent[cur];
        if (up < 0) return;
        __threadfence();
        if (atomicAdd(&arrive[up], 1) != 3) return;
        __threadfence();
        i64 first = node_child[up];
        double xmid = node_center[2 * up], ymid = node_center[2 * up + 1];
        double acc_re[W], acc_im[W];
#pragma unroll
        for (int n = 0; n < W; ++n) acc_re[n] = acc_im[n] = 0.0;
        double qabs = 0.0;
        for (i64 child = first; child < first + 4; ++child) {
            qabs += __ldcg(node_qabs + child);
            if (node_end[child] == node_start[child]) continue;
            double s_re = node_center[2 * child] - xmid;
            double s_im = node_center[2 * child + 1] - ymid;
            double sh_re[W], sh_im[W], cr[W], ci[W];
            sh_re[0] = 1.0;
            sh_im[0] = 0.0;
#pragma unroll
            for (int n = 1; n < W; ++n) {
                sh_re[n] = sh_re[n - 1] * s_re - sh_im[n - 1] * s_im;
                sh_im[n] = sh_re[n - 1] * s_im + sh_im[n - 1] * s_re;
            }
#pragma unroll
            for (int m = 0; m < W; ++m) {
                cr[m] = m < w ? __ldcg(moment_re + child * w + m) : 0.0;
                ci[m] = m < w ? __ldcg(moment_im + child * w + m) : 0.0;
            }
#pragma unroll
            for (int n = 0; n < W; ++n) {
                double c_re = 0.0, c_im = 0.0;
#pragma unroll
                for (int m = 0; m <= n; ++m) {
                    double b = binomial[n * bsize + m];
                    double a_re = cr[m] * b, a_im = ci[m] * b;
                    c_re += a_re * sh_re[n - m] - a_im * sh_im[n - m];
                    c_im += a_re * sh_im[n - m] + a_im * sh_re[n - m];
                }
                acc_re[n] += c_re;
                acc_im[n] += c_im;
            }
        }
#pragma unroll
        for (int n = 0; n < W; ++n) {
            if (n < w) {
                moment_re[up * w + n] = acc_re[n];
                moment_im[up * w + n] = acc_im[n];
            }
        }
        node_qabs[up] = qabs;
        cur = up;
    }
}

// Moments of every node.  Orders up to 15: every leaf in one launch (leaves depend on
// nothing), then the internal nodes level by level, deepest first, a thread per (node,
// child); higher orders: thread per (node, coefficient), level by level.
int launch_log_moments(const int64_t* levels, int64_t n_levels, int order, const double* spos,
                       const double* scharge, int64_t n, const double* center, const i64* start,
                       const i64* end, const i64* child, const double* binomial, int bsize,
                       double* qabs, double* mre, double* mim, const double* sdip,
                       cudaStream_t s) {
    i64 count = levels[n_levels];
    if (count <= 0) return TD3_OK;
    if (order <= 15) {
        unsigned nb = td3_blocks(count, MOM_THREADS);
#define TD3_LEAF_MOMENTS(P)                                                                  \
    TD3_TRY(td3_launch_chained(k_log_leaf_moments<P>, nb, MOM_THREADS, 0, s, count, order, spos, \
                               scharge, n, center, start, end, child, qabs, mre, mim, sdip))
#define TD3_M2M(P)                                                                           \
    TD3_TRY(td3_launch_chained(k_log_m2m_level<P>, nb, M2M_NODES * 4, 0, s, lo, hi, order,    \
                               center, start, end, child, binomial, bsize, qabs, mre, mim))
        if (order <= 4)
            TD3_LEAF_MOMENTS(4);
        else if (order <= 8)
            TD3_LEAF_MOMENTS(8);
        else if (order <= 12)
            TD3_LEAF_MOMENTS(12);
        else
            TD3_LEAF_MOMENTS(15);
        for (i64 level = n_levels - 2; level >= 0; --level) {
            i64 lo = levels[level], hi = levels[level + 1];
            if (hi <= lo) continue;
            nb = (unsigned)((hi - lo + M2M_NODES - 1) / M2M_NODES);
            if (order <= 4)
                TD3_M2M(4);
            else if (order <= 8)
                TD3_M2M(8);
            else if (order <= 12)
                TD3_M2M(12);
            else
                TD3_M2M(15);
        }
#undef TD3_LEAF_MOMENTS
#undef TD3_M2M
    } else {
        for (i64 level = n_levels - 1; level >= 0; --level) {
            i64 lo = levels[level], hi = levels[level + 1];
            if (hi <= lo) continue;
            k_log_moments<<<td3_blocks((hi - lo) * (order + 1), MOM_THREADS), MOM_THREADS, 0,
                            s>>>(lo, hi, order, spos, scharge, n, center, start, end, child,
                                 binomial, bsize, qabs, mre, mim, sdip);
        }
    }
    TD3_CHECK_LAUNCH();
    return TD3_OK;
}

// Cartesian moments with a block per node and thread g per coefficient.  The monomials
// u^(a,b) a particle (or a child's shift) needs are built once into shared memory, column
// b by thread b as the reference's mono recurrence builds them (b factors of u_y, then
// u_x one at a time; for a particle the first factor is its charge), and each
// coefficient sums them row by row in the reference's order.
__device__ __forceinline__ int cart_index(int a, int b) { return (a + b) * (a + b + 1) / 2 + b; }

constexpr int CART_MOM_THREADS = 256;
constexpr int CART_MOM_PER_THREAD = 9;  // 256 x 9 coefficients: orders up to 66

__global__ void __launch_bounds__(CART_MOM_THREADS)
k_cart_moments_block(i64 lo, int order, int n_coef, const double* __restrict__ spos,
                     const double* __restrict__ scharge, i64 n_particles,
                     const double* __restrict__ node_center, const i64* __restrict__ node_start,
                     const i64* __restrict__ node_end, const i64* __restrict__ node_child,
                     const i64* __restrict__ shift, const double* __restrict__ shift_coef,
                     const i64* __restrict__ shift_start, double* moments,
                     const double* __restrict__ sdip) {
    extern __shared__ double mono_tab[];  // [n_coef] start q (or 1), [n_coef] start 1
    i64 node = lo + blockIdx.x;
    double xmid = node_center[2 * node], ymid = node_center[2 * node + 1];
    double acc[CART_MOM_PER_THREAD];
#pragma unroll
    for (int j = 0; j < CART_MOM_PER_THREAD; ++j) acc[j] = 0.0;
    i64 first = node_child[node];
    if (first < 0) {
        for (i64 k = node_start[node]; k < node_end[node]; ++k) {
            double q = scharge[k];
            double ux = spos[k] - xmid, uy = spos[n_particles + k] - ymid;
            __syncthreads();
            for (int dy = threadIdx.x; dy <= order; dy += blockDim.x) {
                double v = q, w = 1.0;
                for (int t = 0; t < dy; ++t) {
                    v = v * uy;
                    w = w * uy;
                }
                for (int dx = 0; dx + dy <= order; ++dx) {
                    mono_tab[cart_index(dx, dy)] = v;
                    if (sdip) mono_tab[n_coef + cart_index(dx, dy)] = w;
                    v = v * ux;
                    w = w * ux;
                }
            }
            __syncthreads();
#pragma unroll
            for (int j = 0; j < CART_MOM_PER_THREAD; ++j) {
                int g = threadIdx.x + j * blockDim.x;
                if (g >= n_coef) break;
                acc[j] += mono_tab[g];
                if (sdip) {
                    int n = 0;
                    while ((n + 1) * (n + 2) / 2 <= g) ++n;
                    int gb = g - n * (n + 1) / 2, ga = n - gb;
                    // a point dipole p = -e: m_g += p . grad (r - c)^g
                    if (ga > 0) acc[j] -= sdip[k] * ga * mono_tab[n_coef + cart_index(ga - 1, gb)];
                    if (gb > 0)
                        acc[j] -= sdip[n_particles + k] * gb *
                                  mono_tab[n_coef + cart_index(ga, gb - 1)];
                }
            }
        }
    } else {
        for (i64 child = first; child < first + 4; ++child) {
            if (node_end[child] == node_start[child]) continue;
            double ux = node_center[2 * child] - xmid, uy = node_center[2 * child + 1] - ymid;
            __syncthreads();
            for (int dy = threadIdx.x; dy <= order; dy += blockDim.x) {
                double v = 1.0;
                for (int t = 0; t < dy; ++t) v = v * uy;
                for (int dx = 0; dx + dy <= order; ++dx) {
                    mono_tab[cart_index(dx, dy)] = v;
                    v = v * ux;
                }
            }
            __syncthreads();
            const double* cm = moments + child * n_coef;
#pragma unroll
            for (int j = 0; j < CART_MOM_PER_THREAD; ++j) {
                int g = threadIdx.x + j * blockDim.x;
                if (g >= n_coef) break;
                for (i64 r = shift_start[g]; r < shift_start[g + 1]; ++r) {
                    int b = (int)shift[3 * r + 1];
                    int d = (int)shift[3 * r + 2];
                    acc[j] += shift_coef[r] * cm[b] * mono_tab[d];
                }
            }
        }
    }
#pragma unroll
    for (int j = 0; j < CART_MOM_PER_THREAD; ++j) {
        int g = threadIdx.x + j * blockDim.x;
        if (g < n_coef) moments[node * n_coef + g] = acc[j];
    }
}

int launch_cart_moments(const int64_t* levels, int64_t n_levels, const double* spos,
                        const double* scharge, int64_t n, const double* center, const i64* start,
                        const i64* end, const i64* child, const i64* shift,
                        const double* shift_coef, const i64* shift_start, int n_coef,
                        double* moments, const double* sdip, cudaStream_t s) {
    int order = 0;
    while ((order + 1) * (order + 2) / 2 < n_coef) ++order;
    if ((order + 1) * (order + 2) / 2 != n_coef) return TD3_EINVAL;
    unsigned threads = (unsigned)((n_coef + 31) / 32 * 32);
    if (threads > CART_MOM_THREADS) threads = CART_MOM_THREADS;
    if (n_coef > (int)threads * CART_MOM_PER_THREAD) return TD3_EINVAL;
    size_t smem = sizeof(double) * 2 * n_coef;
    if (smem > 48 * 1024)
        TD3_TRY(cudaFuncSetAttribute(k_cart_moments_block,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    for (i64 level = n_levels - 1; level >= 0; --level) {
        i64 lo = levels[level], hi = levels[level + 1];
        if (hi <= lo) continue;
        k_cart_moments_block<<<(unsigned)(hi - lo), threads, smem, s>>>(
            lo, order, n_coef, spos, scharge, n, center, start, end, child, shift, shift_coef,
            shift_start, moments, sdip);
    }
    TD3_CHECK_LAUNCH();
    return TD3_OK;
}

}  // namespace

extern "C" int td3_quadtree_moments(const int64_t* levels, int64_t n_levels,
                                    const double* sorted_pos, const double* sorted_charge,
                                    int64_t n, const double* node_center,
                                    const int64_t* node_start, const int64_t* node_end,
                                    const int64_t* node_child, double* node_q, double* node_qabs,
                                    double* node_p, double* node_s, void* stream) {
    if (n_levels < 1) return TD3_EINVAL;
    cudaStream_t s = td3_stream(stream);
    for (i64 level = n_levels - 1; level >= 0; --level) {
        i64 lo = levels[level], hi = levels[level + 1];
        if (hi <= lo) continue;
        k_coulomb_moments<<<td3_blocks(hi - lo, MOM_THREADS), MOM_THREADS, 0, s>>>(
            lo, hi, sorted_pos, sorted_charge, n, node_center, node_start, node_end, node_child,
            node_q, node_qabs, node_p, node_s);
    }
    TD3_CHECK_LAUNCH();
    return TD3_OK;
}

extern "C" int td3_log_moments(const int64_t* levels, int64_t n_levels, int order,
                               const double* sorted_pos, const double* sorted_charge, int64_t n,
                               const double* node_center, const int64_t* node_start,
                               const int64_t* node_end, const int64_t* node_child,
                               const double* binomial, int binomial_size, double* node_qabs,
                               double* moment_re, double* moment_im, void* stream) {
    if (n_levels < 1 || order < 0 || order > TD3_MAX_ORDER || binomial_size < order + 1)
        return TD3_EINVAL;
    return launch_log_moments(levels, n_levels, order, sorted_pos, sorted_charge, n, node_center,
                              node_start, node_end, node_child, binomial, binomial_size,
                              node_qabs, moment_re, moment_im, nullptr, td3_stream(stream));
}

extern "C" int td3_log_moments_adjoint(const int64_t* levels, int64_t n_levels, int order,
                                       const double* sorted_pos, const double* sorted_weight,
                                       const double* sorted_dipole, int64_t n,
                                       const double* node_center, const int64_t* node_start,
                                       const int64_t* node_end, const int64_t* node_child,
                                       const double* binomial, int binomial_size,
                                       double* node_wabs, double* moment_re, double* moment_im,
                                       void* stream) {
    if (n_levels < 1 || order < 0 || order > TD3_MAX_ORDER || binomial_size < order + 1)
        return TD3_EINVAL;
    return launch_log_moments(levels, n_levels, order, sorted_pos, sorted_weight, n, node_center,
                              node_start, node_end, node_child, binomial, binomial_size,
                              node_wabs, moment_re, moment_im, sorted_dipole, td3_stream(stream));
}

extern "C" int td3_cart_moments(const int64_t* levels, int64_t n_levels, const double* sorted_pos,
                                const double* sorted_charge, int64_t n, const double* node_center,
                                const int64_t* node_start, const int64_t* node_end,
                                const int64_t* node_child, const int64_t* ex, const int64_t* ey,
                                const int64_t* shift, const double* shift_coef,
                                const int64_t* shift_start, int n_coef, double* moments,
                                void* stream) {
    if (n_levels < 1 || n_coef < 1) return TD3_EINVAL;
    (void)ex;
    (void)ey;
    return launch_cart_moments(levels, n_levels, sorted_pos, sorted_charge, n, node_center,
                               node_start, node_end, node_child, shift, shift_coef, shift_start,
                               n_coef, moments, nullptr, td3_stream(stream));
}

extern "C" int td3_cart_moments_adjoint(const int64_t* levels, int64_t n_levels,
                                        const double* sorted_pos, const double* sorted_weight,
                                        const double* sorted_dipole, int64_t n,
                                        const double* node_center, const int64_t* node_start,
                                        const int64_t* node_end, const int64_t* node_child,
                                        const int64_t* ex, const int64_t* ey,
                                        const int64_t* shift, const double* shift_coef,
                                        const int64_t* shift_start, int n_coef, double* moments,
                                        void* stream) {
    if (n_levels < 1 || n_coef < 1) return TD3_EINVAL;
    (void)ex;
    (void)ey;
    return launch_cart_moments(levels, n_levels, sorted_pos, sorted_weight, n, node_center,
                               node_start, node_end, node_child, shift, shift_coef, shift_start,
                               n_coef, moments, sorted_dipole, td3_stream(stream));
}

extern "C" int td3_log_moments_tree(int64_t count, int order, const double* sorted_pos,
                                    const double* sorted_charge, const double* sorted_dipole,
                                    int64_t n, const double* node_center,
                                    const int64_t* node_start, const int64_t* node_end,
                                    const int64_t* node_child, const int32_t* node_parent,
                                    const double* binomial, int binomial_size, double* node_qabs,
                                    double* moment_re, double* moment_im, int32_t* arrive,
                                    void* stream) {
    if (count < 1 || count > 0x7fffffffLL || order < 0 || order > 12 ||
        binomial_size < order + 1)
        return TD3_EINVAL;
    cudaStream_t s = td3_stream(stream);
    TD3_TRY(cudaMemsetAsync(arrive, 0, sizeof(int32_t) * count, s));
    unsigned nb = td3_blocks(count, MOM_THREADS);
    if (order <= 4)
        k_log_moments_tree<4><<<nb, MOM_THREADS, 0, s>>>(
            count, order, sorted_pos, sorted_charge, n, node_center, node_start, node_end,
            node_child, node_parent, binomial, binomial_size, node_qabs, moment_re, moment_im,
            sorted_dipole, arrive);
    else if (order <= 8)
        k_log_moments_tree<8><<<nb, MOM_THREADS, 0, s>>>(
            count, order, sorted_pos, sorted_charge, n, node_center, node_start, node_end,
            node_child, node_parent, binomial, binomial_size, node_qabs, moment_re, moment_im,
            sorted_dipole, arrive);
    else
        k_log_moments_tree<12><<<nb, MOM_THREADS, 0, s>>>(
            count, order, sorted_pos, sorted_charge, n, node_center, node_start, node_end,
            node_child, node_parent, binomial, binomial_size, node_qabs, moment_re, moment_im,
            sorted_dipole, arrive);
    TD3_CHECK_LAUNCH();
    return TD3_OK;
}
