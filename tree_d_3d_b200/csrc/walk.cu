// Barnes-Hut walks of both kernels: evaluate_quadtree (K/evaluate_quadtree/
// evaluate_quadtree_cuda.cu:9-107) and evaluate_log_quadtree (K/evaluate_log_quadtree/
// evaluate_log_quadtree_cuda.cu:9-104), whose CPU form is evaluate_groups
// (K/evaluate_groups/evaluate_groups_pyccel.py:16-297).
//
// Warp-cooperative and stackless: a warp takes 32 consecutive targets of a spatial
// order and walks the tree once for all of them, following precomputed "next"
// pointers (the node visited after a node's subtree) in the reference's visiting
// order (children popped 3, 2, 1, 0).  mask[d] (shared memory) holds the lanes that
// opened every ancestor at depth < d; a lane accepts or opens each internal node by
// the reference's test, evaluated with exactly rounded operations (no FMA), so every
// target gets exactly the terms of its own walk, in the same order.  The warp
// descends while any lane needs the children.  Node data is packed per node for
// broadcast loads.
#include "common.cuh"

namespace {

constexpr int WALK_THREADS = 128;
constexpr int WALK_WARPS = WALK_THREADS / 32;
constexpr int MAX_DEPTH_WALK = 190;
constexpr int COULOMB_STRIDE = 10;  // cx, cy, half, qabs, q, px, py, sxx, sxy, syy

__global__ void k_parents(i64 count, const i64* __restrict__ node_child, int* __restrict__ parent) {
    i64 p = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= count) return;
    if (p == 0) parent[0] = -1;
    i64 c = node_child[p];
    if (c >= 0)
        for (int k = 0; k < 4; ++k) parent[c + k] = (int)p;
}

// links = (child, next, start, end); depth as int.  next(n): the sibling visited after
// n (n - 1 unless n is its parent's first child), else next(parent); -1 at the end.
__global__ void k_links(i64 count, const i64* __restrict__ node_child,
                        const i64* __restrict__ node_start, const i64* __restrict__ node_end,
                        const i64* __restrict__ node_depth, const int* __restrict__ parent,
                        int4* __restrict__ links, int* __restrict__ depth) {
    i64 n = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= count) return;
    int next = -1;
    int cur = (int)n;
    while (cur != 0) {
        int p = parent[cur];
        if (cur - (int)node_child[p] > 0) {
            next = cur - 1;
            break;
        }
        cur = p;
    }
    links[n] = make_int4((int)node_child[n], next, (int)node_start[n], (int)node_end[n]);
    depth[n] = (int)node_depth[n];
}

__global__ void k_pack_coulomb(i64 count, const double* __restrict__ center,
                               const double* __restrict__ half, const double* __restrict__ qabs,
                               const double* __restrict__ q, const double* __restrict__ p,
                               const double* __restrict__ s, double* __restrict__ packed) {
    i64 n = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= count) return;
    double* o = packed + n * COULOMB_STRIDE;
    o[0] = center[2 * n];
    o[1] = center[2 * n + 1];
    o[2] = half[n];
    o[3] = qabs[n];
    o[4] = q[n];
    o[5] = p[2 * n];
    o[6] = p[2 * n + 1];
    o[7] = s[3 * n];
    o[8] = s[3 * n + 1];
    o[9] = s[3 * n + 2];
}

__global__ void k_pack_geometry(i64 count, const double* __restrict__ center,
                                const double* __restrict__ half, const double* __restrict__ qabs,
                                double4* __restrict__ packed) {
    i64 n = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= count) return;
    packed[n] = make_double4(center[2 * n], center[2 * n + 1], half[n], qabs[n]);
}

__device__ __forceinline__ bool inside_cell(double tx, double ty, double cx, double cy, double h) {
    return tx >= xsub(cx, h) && tx <= xadd(cx, h) && ty >= xsub(cy, h) && ty <= xadd(cy, h);
}

// The mixed-precision form of the walk (MIXED): the opening decisions are the exactly
// rounded FP64 tests of the FP64 form, so every target takes the same terms; a leaf pair
// forms its difference in FP64 and the kernel in FP32, and a far-field term is evaluated
// in FP32 in units of the distance (Coulomb) or on size-scaled moments (log) so no FP32
// intermediate under- or overflows for small cells.  Terms go into compensated FP32 sums.
template <bool POT, bool MIXED>
__global__ void __launch_bounds__(WALK_THREADS)
k_walk_coulomb(const double* __restrict__ targets, i64 m, const i64* __restrict__ exclude,
               const i64* __restrict__ order, const double* __restrict__ spos,
               const double* __restrict__ scharge, const i64* __restrict__ sindex, i64 n,
               const double* __restrict__ nodes, const int4* __restrict__ links,
               const int* __restrict__ depth, double theta, double eps2, double* __restrict__ phi,
               double* __restrict__ field, i64* status) {
    __shared__ unsigned masks[WALK_WARPS][MAX_DEPTH_WALK + 2];
    int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    i64 t = ((i64)blockIdx.x * WALK_WARPS + wib) * 32 + lane;
    bool valid = t < m;
    i64 i = valid ? (order ? order[t] : t) : 0;
    double tx = valid ? targets[i] : 0.0, ty = valid ? targets[m + i] : 0.0;
    i64 skip = valid ? exclude[i] : -2;
    double pot = 0.0, ex = 0.0, ey = 0.0;
    // MIXED: lengths in units of the root half-width L (FP32 terms O(1) at any scale);
    // the sums are q / r' and q d' / r'^3, so phi = sum / L and E = sum / L^2.
    KahanF kp, kx, ky;
    double unit = nodes[2], inv_unit = 1.0 / unit;
    float eps2f = (float)(eps2 * inv_unit * inv_unit);
    bool bad = false;
    unsigned* mk = masks[wib];
    unsigned active = __ballot_sync(0xffffffffu, valid);
    if (active == 0) return;
    if (lane == 0) mk[0] = active;
    __syncwarp();
    int node = 0;
    while (node >= 0) {
        int d = depth[node];
        bool in = (mk[d] >> lane) & 1u;
        const double* nd = nodes + (i64)node * COULOMB_STRIDE;
        double2 c01 = *reinterpret_cast<const double2*>(nd);
        double2 c23 = *reinterpret_cast<const double2*>(nd + 2);
        int4 L = links[node];
        if (c23.y == 0.0) {  // sum |q| == 0: nothing to add below
            node = L.y;
            continue;
        }
        if (L.x < 0) {
            if (in && !bad) {
                for (int k = L.z; k < L.w; ++k) {
                    double c = scharge[k];
                    if (c == 0.0 || sindex[k] == skip) continue;
                    double dx = tx - spos[k];
                    double dy = ty - spos[n + k];
                    if constexpr (MIXED) {
                        if (dx == 0.0 && dy == 0.0 && eps2 == 0.0) {
                            bad = true;
                            break;
                        }
                        float fx = (float)(dx * inv_unit), fy = (float)(dy * inv_unit);
                        float qf = (float)c;
                        float ir = rsqrtf(fmaf(fx, fx, fmaf(fy, fy, eps2f)));
                        float qr3 = qf * ir * ir * ir;
                        if (POT) kp.add(qf * ir);
                        kx.add(qr3 * fx);
                        ky.add(qr3 * fy);
                        continue;
                    }
                    double r2 = dx * dx + dy * dy + eps2;
                    if (r2 == 0.0) {
                        bad = true;
                        break;
                    }
                    double inv_r = rsqrt(r2);
                    double inv_r3 = inv_r * inv_r * inv_r;
                    pot += c * inv_r;
                    ex += c * inv_r3 * dx;
                    ey += c * inv_r3 * dy;
                }
            }
            node = L.y;
            continue;
        }
        bool open = false;
        if (in) {
            double cx = c01.x, cy = c01.y, h = c23.x;
            double rx = xsub(tx, cx), ry = xsub(ty, cy);
            double d2 = xnorm2(rx, ry);
            double distance = xsqrt(d2);
            if (!inside_cell(tx, ty, cx, cy, h) && xmul(2.0, h) < xmul(theta, distance)) {
                if (!bad && MIXED) {
                    // u = r / rho, p^ = p / rho, S^ = S / rho^2 (rho^2 = |r|^2 + eps^2):
                    // phi = [q + p^.u + (3 u.S^u - tr S^) / 2] / rho and
                    // E = [(q + 3 p^.u + 7.5 u.S^u - 1.5 tr S^) u - p^ - 3 S^u] / rho^2.
                    double2 q45 = *reinterpret_cast<const double2*>(nd + 4);
                    double2 q67 = *reinterpret_cast<const double2*>(nd + 6);
                    double2 q89 = *reinterpret_cast<const double2*>(nd + 8);
                    double ir = rsqrt(d2 + eps2), ir2 = ir * ir;
                    float ux = (float)(rx * ir), uy = (float)(ry * ir);
                    float q = (float)q45.x, px = (float)(q45.y * ir), py = (float)(q67.x * ir);
                    float sxx = (float)(q67.y * ir2), sxy = (float)(q89.x * ir2),
                          syy = (float)(q89.y * ir2);
                    float pr = fmaf(px, ux, py * uy);
                    float srx = fmaf(sxx, ux, sxy * uy), sry = fmaf(sxy, ux, syy * uy);
                    float rsr = fmaf(ux, srx, uy * sry), trace = sxx + syy;
                    double iru = ir * unit;  // 1 / rho in units of L
                    if (POT) kp.add((float)((double)(q + pr + 0.5f * fmaf(3.0f, rsr, -trace)) * iru));
                    float radial = q + 3.0f * pr + 7.5f * rsr - 1.5f * trace;
                    kx.add((float)((double)(fmaf(radial, ux, -px) - 3.0f * srx) * (iru * iru)));
                    ky.add((float)((double)(fmaf(radial, uy, -py) - 3.0f * sry) * (iru * iru)));
                } else if (!bad) {
                    double2 q45 = *reinterpret_cast<const double2*>(nd + 4);
                    double2 q67 = *reinterpret_cast<const double2*>(nd + 6);
                    double2 q89 = *reinterpret_cast<const double2*>(nd + 8);
                    double q = q45.x, px = q45.y, py = q67.x, sxx = q67.y, sxy = q89.x,
                           syy = q89.y;
                    double inv_r = rsqrt(distance * distance + eps2);
                    double inv_r2 = inv_r * inv_r;
                    double inv_r3 = inv_r2 * inv_r;
                    double inv_r5 = inv_r3 * inv_r2;
                    double inv_r7 = inv_r5 * inv_r2;
                    double pr = px * rx + py * ry;
                    double srx = sxx * rx + sxy * ry;
                    double sry = sxy * rx + syy * ry;
                    double rsr = rx * srx + ry * sry;
                    double trace = sxx + syy;
                    pot += q * inv_r + pr * inv_r3 + 0.5 * (3.0 * rsr * inv_r5 - trace * inv_r3);
                    double radial = q * inv_r3 + 3.0 * pr * inv_r5 + 7.5 * rsr * inv_r7 -
                                    1.5 * trace * inv_r5;
                    ex += radial * rx - px * inv_r3 - 3.0 * srx * inv_r5;
                    ey += radial * ry - py * inv_r3 - 3.0 * sry * inv_r5;
                }
            } else {
                open = true;
            }
        }
        unsigned r = __ballot_sync(0xffffffffu, open);
        if (r) {
            if (lane == 0) mk[d + 1] = r;
            __syncwarp();
            node = L.x + 3;
        } else {
            node = L.y;
        }
    }
    if (!valid) return;
    if (bad) td3_report(status, i + 1);
    if constexpr (MIXED) {
        pot = kp.value() * inv_unit;
        ex = kx.value() * inv_unit * inv_unit;
        ey = ky.value() * inv_unit * inv_unit;
    }
    phi[i] = POT ? pot : 0.0;
    field[i] = ex;
    field[m + i] = ey;
}

// hat (MIXED only): the moments scaled by the cell size, hat_k = a_k / h^k as FP32 pairs,
// (order_p + 1) per node.
template <bool POT, bool MIXED>
__global__ void __launch_bounds__(WALK_THREADS)
k_walk_log(const double* __restrict__ targets, i64 m, const i64* __restrict__ exclude,
           const i64* __restrict__ order, const double* __restrict__ spos,
           const double* __restrict__ scharge, const i64* __restrict__ sindex, i64 n,
           const double4* __restrict__ geom, const int4* __restrict__ links,
           const int* __restrict__ depth, const double* __restrict__ moment_re,
           const double* __restrict__ moment_im, const float2* __restrict__ hat, int order_p,
           double theta, double eps2, double* __restrict__ phi, double* __restrict__ field,
           i64* status) {
    __shared__ unsigned masks[WALK_WARPS][MAX_DEPTH_WALK + 2];
    __shared__ double inv_n[TD3_MAX_ORDER + 1];
    __shared__ float inv_nf[TD3_MAX_ORDER + 1];
    for (int k = threadIdx.x; k <= order_p; k += blockDim.x) {
        inv_n[k] = k ? 1.0 / k : 0.0;
        inv_nf[k] = (float)inv_n[k];
    }
    __syncthreads();
    int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    i64 t = ((i64)blockIdx.x * WALK_WARPS + wib) * 32 + lane;
    bool valid = t < m;
    i64 i = valid ? (order ? order[t] : t) : 0;
    double tx = valid ? targets[i] : 0.0, ty = valid ? targets[m + i] : 0.0;
    i64 skip = valid ? exclude[i] : -2;
    double pot = 0.0, ex = 0.0, ey = 0.0;
    // MIXED: lengths in units of the root half-width L: -q ln r^2 = -q ln r'^2 - q ln L^2,
    // the first summed in FP32, the charges of the second (qsum) in FP64; E = sum / L.
    KahanF kp, kx, ky;
    double unit = geom[0].z, inv_unit = 1.0 / unit, inv_unit2 = inv_unit * inv_unit;
    double qsum = 0.0;
    float eps2f = (float)(eps2 * inv_unit2);
    bool bad = false;
    unsigned* mk = masks[wib];
    unsigned active = __ballot_sync(0xffffffffu, valid);
    if (active == 0) return;
    if (lane == 0) mk[0] = active;
    __syncwarp();
    double theta2 = xmul(theta, theta);
    int w = order_p + 1;
    int node = 0;
    while (node >= 0) {
        int d = depth[node];
        bool in = (mk[d] >> lane) & 1u;
        double4 g = geom[node];
        int4 L = links[node];
        if (g.w == 0.0) {
            node = L.y;
            continue;
        }
        if (L.x < 0) {
            if (in && !bad) {
                for (int k = L.z; k < L.w; ++k) {
                    double c = scharge[k];
                    if (c == 0.0 || sindex[k] == skip) continue;
                    double dx = tx - spos[k];
                    double dy = ty - spos[n + k];
                    if constexpr (MIXED) {
                        if (dx == 0.0 && dy == 0.0 && eps2 == 0.0) {
                            bad = true;
                            break;
                        }
                        float fx = (float)(dx * inv_unit), fy = (float)(dy * inv_unit);
                        float qf = (float)c;
                        float r2 = fmaf(fx, fx, fmaf(fy, fy, eps2f));
                        if (POT) {
                            kp.add(-qf * __logf(r2));
                            qsum += c;
                        }
                        float f = __fdividef(2.0f * qf, r2);
                        kx.add(f * fx);
                        ky.add(f * fy);
                        continue;
                    }
                    double r2 = dx * dx + dy * dy + eps2;
                    if (r2 == 0.0) {
                        bad = true;
                        break;
                    }
                    if (POT) pot -= c * log(r2);
                    double f = 2.0 * c / r2;
                    ex += f * dx;
                    ey += f * dy;
                }
            }
            node = L.y;
            continue;
        }
        bool open = false;
        if (in) {
            double rx = xsub(tx, g.x), ry = xsub(ty, g.y);
            double d2 = xnorm2(rx, ry);
            if (!inside_cell(tx, ty, g.x, g.y, g.z) && xmul(xmul(4.0, g.z), g.z) < xmul(theta2, d2)) {
                if (!bad && MIXED) {
                    // w = 1 / conj(r) = (rx, -ry) / |r|^2 and w^ = h w (|w^| < theta / 2):
                    // sum_k a_k w^(k+1) = w sum_k hat_k w^^k and sum_k a_k w^k / k =
                    // sum_k hat_k w^^k / k, both by Horner's rule from the highest order.
                    double inv_d2 = 1.0 / d2;
                    double wr64 = rx * inv_d2, wi64 = -ry * inv_d2;
                    float wr = (float)(wr64 * g.z), wi = (float)(wi64 * g.z);
                    wr64 *= unit;  // w in units of 1 / L
                    wi64 *= unit;
                    const float2* a = hat + (i64)node * td3_hat_width(order_p);
                    float2 top = a[order_p];
                    float gr = top.x, gi = top.y;
                    float sr = top.x * inv_nf[order_p], si = top.y * inv_nf[order_p];
                    for (int k = order_p - 1; k >= 0; --k) {
                        float2 ak = a[k];
                        float nr = fmaf(gr, wr, fmaf(-gi, wi, ak.x));
                        gi = fmaf(gr, wi, fmaf(gi, wr, ak.y));
                        gr = nr;
                        if (POT) {
                            float sk = k ? inv_nf[k] : 0.0f;
                            float mr = fmaf(sr, wr, fmaf(-si, wi, ak.x * sk));
                            si = fmaf(sr, wi, fmaf(si, wr, ak.y * sk));
                            sr = mr;
                        }
                    }
                    // after the k = 0 step s holds sum_{k>=1} hat_k w^^k / k (+ 0 w^^0)
                    float fr = (float)wr64, fi = (float)wi64;
                    float er = fmaf(fr, gr, -fi * gi), ei = fmaf(fr, gi, fi * gr);
                    if (POT) {
                        kp.add(fmaf(-a[0].x, log_split(d2 * inv_unit2), 2.0f * sr));
                        qsum += moment_re[(i64)node * w];
                    }
                    kx.add(2.0f * er);
                    ky.add(-2.0f * ei);
                } else if (!bad) {
                    double inv_d2 = 1.0 / d2;
                    double w_re = rx * inv_d2, w_im = -ry * inv_d2;
                    double prev_re = 1.0, prev_im = 0.0, cur_re = w_re, cur_im = w_im;
                    double f_re = 0.0, f_im = 0.0, series = 0.0;
                    const double* are = moment_re + (i64)node * w;
                    const double* aim = moment_im + (i64)node * w;
                    for (int k = 0; k <= order_p; ++k) {
                        double a_re = are[k], a_im = aim[k];
                        f_re += a_re * cur_re - a_im * cur_im;
                        f_im += a_re * cur_im + a_im * cur_re;
                        if (POT) series += (a_re * prev_re - a_im * prev_im) * inv_n[k];
                        prev_re = cur_re;
                        prev_im = cur_im;
                        double next_re = cur_re * w_re - cur_im * w_im;
                        cur_im = cur_re * w_im + cur_im * w_re;
                        cur_re = next_re;
                    }
                    if (POT) pot += -are[0] * log(d2) + 2.0 * series;
                    ex += 2.0 * f_re;
                    ey -= 2.0 * f_im;
                }
            } else {
                open = true;
            }
        }
        unsigned r = __ballot_sync(0xffffffffu, open);
        if (r) {
            if (lane == 0) mk[d + 1] = r;
            __syncwarp();
            node = L.x + 3;
        } else {
            node = L.y;
        }
    }
    if (!valid) return;
    if (bad) td3_report(status, i + 1);
    if constexpr (MIXED) {
        pot = kp.value() - 2.0 * log(unit) * qsum;
        ex = kx.value() * inv_unit;
        ey = ky.value() * inv_unit;
    }
    phi[i] = POT ? pot : 0.0;
    field[i] = ex;
    field[m + i] = ey;
}

template <bool POT, bool MIXED>
void launch_walk_coulomb(unsigned blocks, cudaStream_t s, const double* targets, i64 m,
                         const i64* exclude, const i64* order, const double* spos,
                         const double* scharge, const i64* sindex, i64 n, const double* nodes,
                         const int4* links, const int* depth, double theta, double eps2,
                         double* phi, double* field, i64* status) {
    k_walk_coulomb<POT, MIXED><<<blocks, WALK_THREADS, 0, s>>>(
        targets, m, exclude, order, spos, scharge, sindex, n, nodes, links, depth, theta, eps2, phi,
        field, status);
}

template <bool POT, bool MIXED>
void launch_walk_log(unsigned blocks, cudaStream_t s, const double* targets, i64 m,
                     const i64* exclude, const i64* order, const double* spos,
                     const double* scharge, const i64* sindex, i64 n, const double4* geom,
                     const int4* links, const int* depth, const double* moment_re,
                     const double* moment_im, const float2* hat, int order_p, double theta,
                     double eps2, double* phi, double* field, i64* status) {
    k_walk_log<POT, MIXED><<<blocks, WALK_THREADS, 0, s>>>(
        targets, m, exclude, order, spos, scharge, sindex, n, geom, links, depth, moment_re,
        moment_im, hat, order_p, theta, eps2, phi, field, status);
}

// ------------------------------------------------------------------ target order
__global__ void k_bbox(const double* __restrict__ targets, i64 m, double* __restrict__ box) {
    // box = (xmin, ymin, xmax, ymax), reduced with one block per grid stride
    __shared__ double s[4][256];
    double v[4] = {INFINITY, INFINITY, -INFINITY, -INFINITY};
    for (i64 k = (i64)blockIdx.x * blockDim.x + threadIdx.x; k < m; k += (i64)gridDim.x * blockDim.x) {
        double x = targets[k], y = targets[m + k];
        v[0] = fmin(v[0], x);
        v[1] = fmin(v[1], y);
        v[2] = fmax(v[2], x);
        v[3] = fmax(v[3], y);
    }
    for (int c = 0; c < 4; ++c) s[c][threadIdx.x] = v[c];
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            s[0][threadIdx.x] = fmin(s[0][threadIdx.x], s[0][threadIdx.x + w]);
            s[1][threadIdx.x] = fmin(s[1][threadIdx.x], s[1][threadIdx.x + w]);
            s[2][threadIdx.x] = fmax(s[2][threadIdx.x], s[2][threadIdx.x + w]);
            s[3][threadIdx.x] = fmax(s[3][threadIdx.x], s[3][threadIdx.x + w]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        box[4 * blockIdx.x] = s[0][0];
        box[4 * blockIdx.x + 1] = s[1][0];
        box[4 * blockIdx.x + 2] = s[2][0];
        box[4 * blockIdx.x + 3] = s[3][0];
    }
}

__device__ __forceinline__ unsigned spread16(unsigned v) {
    v = (v | (v << 8)) & 0x00FF00FFu;
    v = (v | (v << 4)) & 0x0F0F0F0Fu;
    v = (v | (v << 2)) & 0x33333333u;
    v = (v | (v << 1)) & 0x55555555u;
    return v;
}

// The reference's target key (ft:891-912): cells = (t - lo) * (65535 / span) truncated,
// x bits at odd positions, y bits at even ones.
__global__ void k_morton(const double* __restrict__ targets, i64 m, const double* __restrict__ box,
                         int n_boxes, unsigned* __restrict__ keys, unsigned* __restrict__ vals) {
    i64 k = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= m) return;
    double lox = INFINITY, loy = INFINITY, hix = -INFINITY, hiy = -INFINITY;
    for (int b = 0; b < n_boxes; ++b) {
        lox = fmin(lox, box[4 * b]);
        loy = fmin(loy, box[4 * b + 1]);
        hix = fmax(hix, box[4 * b + 2]);
        hiy = fmax(hiy, box[4 * b + 3]);
    }
    double span = fmax(hix - lox, hiy - loy);
    double scale = span > 0.0 ? 65535.0 / span : 0.0;
    unsigned cx = (unsigned)(unsigned long long)((targets[k] - lox) * scale);
    unsigned cy = (unsigned)(unsigned long long)((targets[m + k] - loy) * scale);
    keys[k] = (spread16(cx & 0xffffu) << 1) | spread16(cy & 0xffffu);
    vals[k] = (unsigned)k;
}

__global__ void k_widen(const unsigned* __restrict__ in, i64 m, i64* __restrict__ out) {
    i64 k = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < m) out[k] = in[k];
}

constexpr int BBOX_BLOCKS = 64;

}  // namespace

extern "C" size_t td3_target_order_workspace_size(int64_t m) {
    return td3_ws_bytes<double>(4 * BBOX_BLOCKS) + 4 * td3_ws_bytes<unsigned>(m) +
           td3_sort_workspace(m);
}

extern "C" int td3_target_order(const double* targets, int64_t m, int64_t* order, void* workspace,
                                size_t workspace_bytes, void* stream) {
    if (m < 0 || m > 0x7fffffffLL) return TD3_EINVAL;
    if (m == 0) return TD3_OK;
    cudaStream_t s = td3_stream(stream);
    Workspace w(workspace, workspace_bytes);
    double* box = w.take<double>(4 * BBOX_BLOCKS);
    unsigned* k0 = w.take<unsigned>(m);
    unsigned* k1 = w.take<unsigned>(m);
    unsigned* v0 = w.take<unsigned>(m);
    unsigned* v1 = w.take<unsigned>(m);
    if (!v1) return TD3_EWORKSPACE;
    k_bbox<<<BBOX_BLOCKS, 256, 0, s>>>(targets, m, box);
    k_morton<<<td3_blocks(m, 256), 256, 0, s>>>(targets, m, box, BBOX_BLOCKS, k0, v0);
    TD3_CHECK_LAUNCH();
    unsigned *ko, *vo;
    TD3_TRY_RC(td3_radix_sort_u32(k0, k1, v0, v1, m, 32, &ko, &vo, w.base + w.used, w.size - w.used, s));
    k_widen<<<td3_blocks(m, 256), 256, 0, s>>>(vo, m, order);
    TD3_CHECK_LAUNCH();
    return TD3_OK;
}

extern "C" size_t td3_walk_workspace_size(int64_t node_count, int kernel) {
    size_t packed = kernel == TD3_KERNEL_LOG ? td3_ws_bytes<double4>(node_count)
                                             : td3_ws_bytes<double>(COULOMB_STRIDE * node_count);
    return packed + td3_ws_bytes<int4>(node_count) + 2 * td3_ws_bytes<int>(node_count);
}

extern "C" int td3_evaluate_quadtree(int kernel, const double* targets, int64_t m,
                                     const int64_t* exclude, const int64_t* order,
                                     const double* sorted_pos, const double* sorted_charge,
                                     const int64_t* perm, int64_t n, int64_t node_count,
                                     const double* node_center, const double* node_half,
                                     const int64_t* node_start, const int64_t* node_end,
                                     const int64_t* node_child, const int64_t* node_depth,
                                     int64_t tree_depth, const double* node_q, const double* node_qabs,
                                     const double* node_p, const double* node_s,
                                     const double* moment_re, const double* moment_im,
                                     const float* moment_hat, int order_p, double theta,
                                     double softening, int with_potential, int mixed, double* phi,
                                     double* field, int64_t* status, void* workspace,
                                     size_t workspace_bytes, void* stream) {
    if (m < 0 || n < 0 || node_count < 1 || node_count > 0x7fffffffLL || n > 0x7fffffffLL)
        return TD3_EINVAL;
    if (kernel != TD3_KERNEL_COULOMB && kernel != TD3_KERNEL_LOG) return TD3_EINVAL;
    if (kernel == TD3_KERNEL_LOG && (order_p < 0 || order_p > TD3_MAX_ORDER)) return TD3_EINVAL;
    if (kernel == TD3_KERNEL_LOG && mixed && !moment_hat) return TD3_EINVAL;
    if (tree_depth < 0) return TD3_EINVAL;
    if (tree_depth > MAX_DEPTH_WALK) return TD3_EDEPTH;
    if (m == 0) return TD3_OK;
    cudaStream_t s = td3_stream(stream);
    Workspace w(workspace, workspace_bytes);
    void* packed = kernel == TD3_KERNEL_LOG ? (void*)w.take<double4>(node_count)
                                            : (void*)w.take<double>(COULOMB_STRIDE * node_count);
    int4* links = w.take<int4>(node_count);
    int* depth = w.take<int>(node_count);
    int* parent = w.take<int>(node_count);
    if (!parent) return TD3_EWORKSPACE;
    unsigned nb = td3_blocks(node_count, 256);
    k_parents<<<nb, 256, 0, s>>>(node_count, node_child, parent);
    k_links<<<nb, 256, 0, s>>>(node_count, node_child, node_start, node_end, node_depth, parent,
                               links, depth);
    unsigned tb = td3_blocks(m, WALK_THREADS);
    double eps2 = softening * softening;
    if (kernel == TD3_KERNEL_COULOMB) {
        double* pk = static_cast<double*>(packed);
        k_pack_coulomb<<<nb, 256, 0, s>>>(node_count, node_center, node_half, node_qabs, node_q,
                                          node_p, node_s, pk);
        auto go = with_potential ? (mixed ? launch_walk_coulomb<true, true>
                                          : launch_walk_coulomb<true, false>)
                                 : (mixed ? launch_walk_coulomb<false, true>
                                          : launch_walk_coulomb<false, false>);
        go(tb, s, targets, m, exclude, order, sorted_pos, sorted_charge, perm, n, pk, links, depth,
           theta, eps2, phi, field, status);
    } else {
        double4* g = static_cast<double4*>(packed);
        k_pack_geometry<<<nb, 256, 0, s>>>(node_count, node_center, node_half, node_qabs, g);
        auto go = with_potential ? (mixed ? launch_walk_log<true, true> : launch_walk_log<true, false>)
                                 : (mixed ? launch_walk_log<false, true>
                                          : launch_walk_log<false, false>);
        go(tb, s, targets, m, exclude, order, sorted_pos, sorted_charge, perm, n, g, links, depth,
           moment_re, moment_im, reinterpret_cast<const float2*>(moment_hat), order_p, theta, eps2,
           phi, field, status);
    }
    TD3_CHECK_LAUNCH();
    return TD3_OK;
}
