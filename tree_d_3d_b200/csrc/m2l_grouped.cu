// The mixed-precision M2L of the log kernel as dense tensor-core products grouped by
// translation (tcgen05.mma kind tf32, 3xTF32), for the mutual lists of one tree (fmm at
// the sources), orders up to 14.
//
// Reference: fmm_m2l_host (K/fmm_m2l_host/fmm_m2l_host_pyccel.py:16-105) with
// _m2l_coefficients (src/tree_d_3d/flat_tree.py:234-245): t = c_dst - c_src, w = 1/t,
//   a'_k = a_k w^k,  s_l = sum_k coeff[k, l] a'_k,
//   b_0 += a_0 ln t - s_0,  b_l += -(-1)^l s_l w^l.
// On expansions scaled by the cell sizes (hat_k = a_k / h_src^k, bhat_l = b_l h_dst^l),
// with z = t / h_dst and rho = h_src / h_dst, one translation is a fixed complex matrix
//   bhat_l = sum_k T_lk hat_k,
//   T_lk = -(-1)^l coeff[k, l] rho^k z^-(k+l)        (l >= 1),
//   T_0k = -coeff[k, 0] rho^k z^-k + [k = 0] ln|z|,
// plus a_0 ln h_dst, added to b_0 in FP64 (only Re ln t reaches phi and E for real
// charges).  In a tree built by halving, the centres of two cells whose depths differ
// by dl lie on the lattice of the smaller half-width, t = u h_min with integer u, so T
// depends on the key (dl, u) alone.  Every key's T is made once (FP64, split into TF32
// hi + lo) as a 32 x 32 real matrix B: output row 2l + c, input column 2k + c' (c, c' =
// real, imaginary; the interleaving of the scaled-moment rows), and rows 30 and 31 that
// copy a_0 for the ln h_dst term.
//
// Grouping.  Destination cells are ordered, within each depth, by their quadrant in
// their parent (all upper-left children in parent order, then upper-right, lower-left,
// lower-right: cells in the same quadrant of neighbouring parents see the same offsets)
// and cut into tiles of 128.  The directed translations are sorted by (tile, key): a
// (tile, key) run holds at most one translation per destination, so it is one product
// D = A B^T of 128 rows, row m of A the scaled moments of destination m's partner at
// that key (zero if it has none).  A tile's CTA sums its runs' products per destination
// in FP64, in the runs' order (deterministic sums), and adds them to the locals once.
// Translations off the operator table (depth differences beyond one, offsets beyond
// the table, centres off the lattice) sort last in their tile and take the
// per-translation FP32 formula on the CUDA cores of the same CTA.
//
// Per CTA (one tile, 4 warps, one row of the tile per thread):
//   produce: the source rows of a run are fetched by cp.async (16-byte pieces issued by
//     the thread of each translation, into the destination's row of a shared-memory
//     stage) and the key's B (8 KB) by one bulk copy, all counted on the stage's
//     mbarrier (an arrival per thread and the bulk copy's bytes); stages run up to
//     G_STAGES - 1 runs ahead;
//   consume: each thread splits its row into TF32 hi + lo and writes it to tensor
//     memory (tcgen05.st; or to shared memory in the canonical operand layout, the
//     shared-memory form), then one thread issues D = A_hi [B_hi; B_lo]^T (64 columns)
//     and D[:, 0:32] += A_lo B_hi^T (M = 128, K = 32 as four steps of 8) into a fresh D
//     and commits them to an mbarrier; A and D are double-buffered, so the next run's
//     rows go in while the products run, and each run's D[:, 0:32] + D[:, 32:64] is
//     added to the row's FP64 sums (one rounding of FP32 partial sums per run);
//   finish: the off-table translations and the FP64 locals.
// Every wait is bounded (a status word and a drain of the copies and products in
// flight before the CTA releases its tensor memory).
#include "common.cuh"
#include "tcgen05.cuh"

namespace {

constexpr int G_THREADS = 128;
constexpr int G_STAGES = 4;
constexpr int G_B_BYTES = 8192;   // one key: 64 rows (B_hi, B_lo) x 32 columns of TF32
constexpr int G_LBO = 128;        // bytes between core matrices along K
constexpr int G_SBO = 1024;       // bytes between groups of 8 rows (K = 32)
constexpr int G_TMEM_COLS = 256;  // D buffers [0, 64), [64, 128); A buffers [128, 192), [192, 256)
constexpr int G_D_COL = 0;
constexpr int G_A_COL = 128;
constexpr int G_MAX_LEVELS = 64;
constexpr int G_MAX_SPAN = 40;
constexpr uint32_t G_WAIT = 1u << 24;
// output columns 30 and 31 copy a_0 (for the a_0 ln h_dst term): free for every order up
// to 14, whose 2 (order + 1) outputs take columns 0..29
constexpr int G_A0_ROW = 30;

// The first node of every depth (start[n] = the node count), for the quadrant order.
struct GLevels {
    i64 start[G_MAX_LEVELS + 1];
    int n;
};

template <int P>
struct GCoef {
    float c[(P + 1) * (P + 1)];
};

// Bytes between the rows of a shared-memory stage: the row itself (a multiple of 16),
// plus 16 when its count of 16-byte chunks is even, so that the 8 lanes of a quarter
// warp reading chunk c of 8 consecutive rows hit 8 different bank groups.
__host__ __device__ constexpr int stage_stride(int row_bytes) {
    return ((row_bytes / 16) & 1) ? row_bytes : row_bytes + 16;
}

template <int P>
struct GShape {
    static constexpr int HW = (P + 2) & ~1;  // pairs per scaled-moment row
    static constexpr int ROW = HW * 8;
    static constexpr int STRIDE = stage_stride(ROW);
    static constexpr int STAGE_A = G_THREADS * STRIDE;
    // dynamic shared memory: B stages, A stages, [shared-memory A operands], flags
    static constexpr int OFF_B = 0;
    static constexpr int OFF_A = OFF_B + G_STAGES * G_B_BYTES;
    static constexpr int OFF_OP = (OFF_A + G_STAGES * STAGE_A + 1023) & ~1023;
    static constexpr int OP_BYTES = 2 * 2 * G_THREADS * 32 * 4;  // 2 buffers x (hi, lo)
    static constexpr int flags_at(bool smem_a) { return smem_a ? OFF_OP + OP_BYTES : OFF_OP; }
    static constexpr int bytes(bool smem_a) { return flags_at(smem_a) + G_STAGES * G_THREADS + 256; }
};

__device__ __forceinline__ int level_of(const GLevels& L, i64 node) {
    int lo = 0, hi = L.n - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (L.start[mid] <= node) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Position of `node` in the quadrant order (a permutation within each depth; the root
// level, of one node, keeps its place).
__device__ __forceinline__ i64 quad_pos(const GLevels& L, i64 node) {
    int lv = level_of(L, node);
    i64 s = L.start[lv], size = L.start[lv + 1] - s, off = node - s;
    if (size & 3) return node;
    return s + (off & 3) * (size >> 2) + (off >> 2);
}

__device__ __forceinline__ i64 node_at(const GLevels& L, i64 qp) {
    int lv = level_of(L, qp);
    i64 s = L.start[lv], size = L.start[lv + 1] - s, off = qp - s;
    if (size & 3) return qp;
    i64 quarter = size >> 2;
    return s + 4 * (off % quarter) + off / quarter;
}

__host__ __device__ inline int span_side(int span) { return 2 * span + 1; }
__host__ __device__ inline unsigned n_keys(int span) {
    return 3u * (unsigned)(span_side(span) * span_side(span));
}

// ------------------------------------------------------------------ sort keys
// One thread per directed translation e (pair e / 2, destination = its first cell for
// even e, its second for odd e): key (tile, operator key) and value (source << 7 | row).
__global__ void k_group_keys(const i64* __restrict__ pairs, i64 n_pairs,
                             const double* __restrict__ center, const double* __restrict__ half,
                             const i64* __restrict__ depth, GLevels L, int span, int key_bits,
                             unsigned* __restrict__ keys, unsigned* __restrict__ vals) {
    i64 e = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= 2 * n_pairs) return;
    i64 a = pairs[2 * (e >> 1)], b = pairs[2 * (e >> 1) + 1];
    i64 d = (e & 1) ? b : a, s = (e & 1) ? a : b;
    i64 dl = depth[s] - depth[d];
    double hd = half[d], hs = half[s], hmin = hs < hd ? hs : hd;
    double ux = (center[2 * d] - center[2 * s]) / hmin;
    double uy = (center[2 * d + 1] - center[2 * s + 1]) / hmin;
    double rx = rint(ux), ry = rint(uy);
    int side = span_side(span);
    unsigned key = n_keys(span);  // off the table
    if (dl >= -1 && dl <= 1 && fabs(ux - rx) <= 1e-9 && fabs(uy - ry) <= 1e-9 &&
        fabs(rx) <= span && fabs(ry) <= span)
        key = (unsigned)(((int)(dl + 1) * side + (int)rx + span) * side + (int)ry + span);
    i64 qp = quad_pos(L, d);
    keys[e] = ((unsigned)(qp >> 7) << key_bits) | key;
    vals[e] = ((unsigned)s << 7) | (unsigned)(qp & 127);
}

// flag[i] = 1 where a (tile, key) run starts in the sorted keys.
__global__ void k_run_flags(const unsigned* __restrict__ keys, i64 e, int* __restrict__ flag) {
    i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= e) return;
    flag[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1 : 0;
}

// Run starts and the first run of every tile, from the exclusive scan of the flags:
// thread i < e writes its run's start; thread e closes the lists.
__global__ void k_run_emit(const unsigned* __restrict__ keys, const int* __restrict__ flag,
                           const int* __restrict__ rank, const int* __restrict__ n_runs, i64 e,
                           int key_bits, i64 n_tiles, int* __restrict__ tile_run,
                           int* __restrict__ run_start) {
    i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i > e) return;
    if (i == e) {
        int total = *n_runs;
        run_start[total] = (int)e;
        i64 last = e ? (i64)(keys[e - 1] >> key_bits) : -1;
        for (i64 t = last + 1; t <= n_tiles; ++t) tile_run[t] = total;
        return;
    }
    if (!flag[i]) return;
    int r = rank[i];
    run_start[r] = (int)i;
    i64 prev = i ? (i64)(keys[i - 1] >> key_bits) : -1;
    i64 cur = (i64)(keys[i] >> key_bits);
    for (i64 t = prev + 1; t <= cur; ++t) tile_run[t] = r;
}

// ------------------------------------------------------------------ operator table
// Byte offset of element (row, k) of a key's B in the K-major, unswizzled layout.
__host__ __device__ inline int op_offset(int row, int k) {
    return (row >> 3) * G_SBO + (k >> 2) * G_LBO + (row & 7) * 16 + (k & 3) * 4;
}

// One thread per (key, output row n < 32, input column k < 32); writes B_hi at row n and
// B_lo at row n + 32 of the key's 8 KB block.
__global__ void k_m2l_operators(int order, const double* __restrict__ coeff, int span,
                                float* __restrict__ ops) {
    i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    int side = span_side(span);
    if (t >= (i64)n_keys(span) * 1024) return;
    i64 key = t >> 10;
    int n = (int)((t >> 5) & 31), k = (int)(t & 31);
    int dl = (int)(key / (side * side)) - 1, rem = (int)(key % (side * side));
    int ux = rem / side - span, uy = rem % side - span;
    // z = t / h_dst = u h_min / h_dst; rho = h_src / h_dst = 2^-dl
    double f = dl >= 0 ? ldexp(1.0, -dl) : 1.0;
    double zr = ux * f, zi = uy * f, z2 = zr * zr + zi * zi;
    int W = order + 1;
    double v = 0.0;
    if (z2 >= 1.0) {
        if (n < 2 * W) {
            int l = n >> 1, co = n & 1, j = k >> 1, ci = k & 1;
            if (j < W) {
                double wr = zr / z2, wi = -zi / z2, pr = 1.0, pi = 0.0;
                for (int m = 0; m < j + l; ++m) {
                    double nr = pr * wr - pi * wi;
                    pi = pr * wi + pi * wr;
                    pr = nr;
                }
                double c = coeff[j * W + l] * ldexp(1.0, -dl * j);
                double sign = l == 0 ? -1.0 : ((l & 1) ? 1.0 : -1.0);
                double tr = sign * c * pr, ti = sign * c * pi;
                if (l == 0 && j == 0) tr += 0.5 * log(z2);
                v = co == 0 ? (ci == 0 ? tr : -ti) : (ci == 0 ? ti : tr);
            }
        } else if (n == G_A0_ROW) {
            v = k == 0 ? 1.0 : 0.0;
        } else if (n == G_A0_ROW + 1) {
            v = k == 1 ? 1.0 : 0.0;
        }
    }
    float hi = td3tc::to_tf32((float)v);
    float lo = td3tc::to_tf32((float)(v - (double)hi));
    unsigned char* base = reinterpret_cast<unsigned char*>(ops) + key * G_B_BYTES;
    *reinterpret_cast<float*>(base + op_offset(n, k)) = hi;
    *reinterpret_cast<float*>(base + op_offset(n + 32, k)) = lo;
}

// ------------------------------------------------------------------ products
// Byte offset of element (row, k) of a 128 x 32 shared-memory A operand.
__device__ __forceinline__ int a_offset(int row, int k) {
    return (row >> 3) * G_SBO + (k >> 2) * G_LBO + (row & 7) * 16 + (k & 3) * 4;
}

// The per-translation FP32 formula (as k_m2l_mixed) for one off-table translation into
// destination d, added to v (bhat_l in v[2l], v[2l + 1]; a_0 in v[2w], v[2w + 1]).
template <int P>
__device__ __forceinline__ void offtable_translation(float (&v)[32], i64 d, i64 src, int order,
                                                     const double* __restrict__ center,
                                                     const double* __restrict__ half,
                                                     const float2* __restrict__ hat,
                                                     const GCoef<P>& C) {
    constexpr int W = P + 1;
    const int w = order + 1;
    double tr = center[2 * d] - center[2 * src], ti = center[2 * d + 1] - center[2 * src + 1];
    double t2 = tr * tr + ti * ti, inv = 1.0 / t2, hd = half[d], hs = half[src];
    float wsr = (float)(hs * tr * inv), wsi = (float)(-hs * ti * inv);
    float wdr = (float)(hd * tr * inv), wdi = (float)(-hd * ti * inv);
    float lnt = 0.5f * log_split(t2 / (hd * hd));
    const float2* row = hat + src * td3_hat_width(order);
    float ar[W], ai[W];
    float pr = 1.0f, pi = 0.0f;
#pragma unroll
    for (int k = 0; k < W; ++k) {
        float2 m = k < w ? row[k] : make_float2(0.0f, 0.0f);
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
        if (l < w) {
            if (l == 0) {
                v[0] += ar[0] * lnt - sr;
                v[1] += ai[0] * lnt - si;
            } else {
                float sign = (l & 1) ? 1.0f : -1.0f;
                v[2 * l] += sign * (sr * qr - si * qi);
                v[2 * l + 1] += sign * (sr * qi + si * qr);
            }
        }
        float nr = qr * wdr - qi * wdi;
        qi = qr * wdi + qi * wdr;
        qr = nr;
    }
    v[G_A0_ROW] += ar[0];
    v[G_A0_ROW + 1] += ai[0];
}

// This thread's row of a run's D (64 columns at taddr): D[:, 0:32] + D[:, 32:64] (the
// second half a correction about 2^-11 of the first, added in FP32) added to the FP64
// sums, for the columns an order up to P uses (when the row took part in the run).
template <int P, int V>
__device__ __forceinline__ void read_out(uint32_t taddr, bool use, double (&acc)[V]) {
    float d0[32], d1[32];
    td3tc::tmem_load32(taddr, d0);
    td3tc::tmem_load32(taddr + 32, d1);
    if (use) {
#pragma unroll
        for (int k = 0; k < V; ++k)
            if (k < 2 * (P + 1) || k >= G_A0_ROW) acc[k] += (double)(d0[k] + d1[k]);
    }
}

template <int P, bool SMEM_A>
__global__ void __launch_bounds__(G_THREADS, SMEM_A ? 1 : 2)
k_m2l_grouped(const int* __restrict__ tile_run, const int* __restrict__ run_start,
              const unsigned* __restrict__ keys, const unsigned* __restrict__ vals, i64 n_nodes,
              GLevels L, const double* __restrict__ center, const double* __restrict__ half,
              const float2* __restrict__ hat, int order, const float* __restrict__ ops,
              int key_bits, unsigned offtable_key, const GCoef<P> C,
              double* __restrict__ local_re, double* __restrict__ local_im, i64* status) {
    using S = GShape<P>;
    constexpr int V = 32;  // outputs per row: bhat_l (re, im) in 0..2P+1, a_0 in 30, 31
    extern __shared__ __align__(1024) unsigned char smem[];
    const int tid = threadIdx.x, warp = tid >> 5;
    const int tile = blockIdx.x;
    const int j0 = tile_run[tile], j1 = tile_run[tile + 1];
    if (j0 == j1) return;
    const unsigned key_mask = (1u << key_bits) - 1u;
    const int jm = (keys[run_start[j1 - 1]] & key_mask) == offtable_key ? j1 - 1 : j1;
    const int n_mma = jm - j0;
    const int w = order + 1, hw = td3_hat_width(order);
    const int chunks = hw / 2;  // 16-byte chunks of a row

    unsigned char* stage_b = smem + S::OFF_B;
    unsigned char* stage_a = smem + S::OFF_A;
    unsigned char* op_a = smem + S::OFF_OP;  // shared-memory A operands (SMEM_A)
    unsigned char* live = smem + S::flags_at(SMEM_A);
    uint64_t* bar_stage = reinterpret_cast<uint64_t*>(live + G_STAGES * G_THREADS);
    uint64_t* bar_mma = bar_stage + G_STAGES;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bar_mma + 2);

    if (tid == 0) {
        // a stage completes when every thread's row copies have landed (one arrival per
        // thread) and the key's B (bytes) is in
        for (int s = 0; s < G_STAGES; ++s) td3tc::mbar_init(&bar_stage[s], G_THREADS);
        td3tc::mbar_init(&bar_mma[0], 1);
        td3tc::mbar_init(&bar_mma[1], 1);
    }
    for (int i = tid; i < G_STAGES * G_THREADS; i += G_THREADS) live[i] = 0;
    if (warp == 0) td3tc::tmem_alloc(tmem_slot, G_TMEM_COLS);
    td3tc::fence_before_sync();
    __syncthreads();
    td3tc::fence_after_sync();
    const uint32_t tmem = *tmem_slot;
    const uint32_t lane_base = (uint32_t)(32 * warp) << 16;

    // run j0 + i into stage i % G_STAGES: the rows by cp.async (each by the thread of its
    // translation), B by one bulk copy; every thread arrives once
    auto produce = [&](int i) {
        int s = i % G_STAGES, j = j0 + i;
        int a = run_start[j], cnt = run_start[j + 1] - a;
        if (tid == 0) {
            unsigned key = keys[a] & key_mask;
            td3tc::mbar_expect_tx(&bar_stage[s], G_B_BYTES);
            td3tc::bulk_g2s(stage_b + s * G_B_BYTES, ops + (size_t)key * (G_B_BYTES / 4), G_B_BYTES,
                            &bar_stage[s]);
        }
        if (tid < cnt) {
            unsigned v = vals[a + tid];
            unsigned m = v & 127u;
            live[s * G_THREADS + m] = 1;
            const unsigned char* src =
                reinterpret_cast<const unsigned char*>(hat + (size_t)(v >> 7) * hw);
            unsigned char* dst = stage_a + s * S::STAGE_A + m * S::STRIDE;
            for (int c = 0; c < chunks; ++c) td3tc::cp_async16(dst + 16 * c, src + 16 * c);
        }
        td3tc::cp_async_arrive(&bar_stage[s]);
    };

    double acc[V];
#pragma unroll
    for (int k = 0; k < V; ++k) acc[k] = 0.0;
    bool failed = false, warp_failed = false, touched = false, prev_live = false;
    int produced = 0, issued = 0;
    const int pre = n_mma < G_STAGES - 1 ? n_mma : G_STAGES - 1;
    for (; produced < pre; ++produced) produce(produced);

    // D of run i in columns [64 (i & 1), +64); A of run i in [128 + 64 (i & 1), +64)

    for (int i = 0; i < n_mma; ++i) {
        const int s = i % G_STAGES;
        bool ok = td3tc::mbar_wait(&bar_stage[s], (uint32_t)(i / G_STAGES) & 1u, G_WAIT);
        // this thread's row: split into TF32 hi + lo
        float hi[32], lo[32];
        const bool is_live = ok && live[s * G_THREADS + tid] != 0;
        touched |= is_live;
        const float4* row = reinterpret_cast<const float4*>(stage_a + s * S::STAGE_A + tid * S::STRIDE);
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            float4 q = (is_live && c < chunks) ? row[c] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            float x[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                hi[4 * c + u] = td3tc::to_tf32(x[u]);
                lo[4 * c + u] = td3tc::to_tf32(x[u] - hi[4 * c + u]);
            }
        }
        if (SMEM_A) {
            unsigned char* ah = op_a + (i & 1) * (2 * G_THREADS * 128);
            unsigned char* al = ah + G_THREADS * 128;
#pragma unroll
            for (int c = 0; c < 8; ++c) {
                *reinterpret_cast<float4*>(ah + a_offset(tid, 4 * c)) =
                    make_float4(hi[4 * c], hi[4 * c + 1], hi[4 * c + 2], hi[4 * c + 3]);
                *reinterpret_cast<float4*>(al + a_offset(tid, 4 * c)) =
                    make_float4(lo[4 * c], lo[4 * c + 1], lo[4 * c + 2], lo[4 * c + 3]);
            }
            td3tc::fence_smem_for_async();
        } else {
            const uint32_t acol = G_A_COL + 64 * (i & 1);
            td3tc::tmem_store32(tmem + lane_base + acol, hi);
            td3tc::tmem_store32(tmem + lane_base + acol + 32, lo);
            td3tc::tmem_wait_st();
        }
        live[s * G_THREADS + tid] = 0;
        td3tc::fence_before_sync();
        if (__syncthreads_or(!ok || warp_failed)) {  // one decision for the whole block
            failed = true;
            break;
        }
        td3tc::fence_after_sync();
        if (tid == 0) {
            constexpr uint32_t id64 = td3tc::idesc_tf32(G_THREADS, 64);
            constexpr uint32_t id32 = td3tc::idesc_tf32(G_THREADS, 32);
            const uint32_t bb = td3tc::smem_addr(stage_b + s * G_B_BYTES);
            const uint32_t d = tmem + G_D_COL + 64 * (i & 1);
#pragma unroll
            for (int ks = 0; ks < 4; ++ks) {
                uint64_t db = td3tc::smem_desc(bb + 2 * G_LBO * ks, G_LBO, G_SBO);
                uint32_t accum = ks > 0 ? 1u : 0u;  // a fresh D for every run
                if (SMEM_A) {
                    uint64_t da = td3tc::smem_desc(
                        td3tc::smem_addr(op_a + (i & 1) * (2 * G_THREADS * 128)) + 2 * G_LBO * ks,
                        G_LBO, G_SBO);
                    td3tc::mma_tf32(d, da, db, id64, accum);
                } else {
                    td3tc::mma_tf32_ts(d, tmem + G_A_COL + 64 * (i & 1) + 8 * ks, db, id64, accum);
                }
            }
#pragma unroll
            for (int ks = 0; ks < 4; ++ks) {
                uint64_t db = td3tc::smem_desc(bb + 2 * G_LBO * ks, G_LBO, G_SBO);
                if (SMEM_A) {
                    uint64_t da = td3tc::smem_desc(
                        td3tc::smem_addr(op_a + (i & 1) * (2 * G_THREADS * 128) + G_THREADS * 128) +
                            2 * G_LBO * ks,
                        G_LBO, G_SBO);
                    td3tc::mma_tf32(d, da, db, id32, 1u);
                } else {
                    td3tc::mma_tf32_ts(d, tmem + G_A_COL + 64 * (i & 1) + 32 + 8 * ks, db, id32,
                                       1u);
                }
            }
            td3tc::mma_commit(&bar_mma[i & 1]);
        }
        issued = i + 1;
        // the previous run: its products are done, its D is summed in FP64 and its stage
        // (whose B they read) takes the next run
        if (i >= 1) {
            bool done = td3tc::mbar_wait(&bar_mma[(i - 1) & 1], (uint32_t)((i - 1) >> 1) & 1u, G_WAIT);
            done = __all_sync(0xffffffffu, done);
            if (done) {
                td3tc::fence_after_sync();
                read_out<P, V>(tmem + lane_base + G_D_COL + 64 * ((i - 1) & 1), prev_live, acc);
            } else {
                warp_failed = true;
            }
        }
        prev_live = is_live;
        if (produced < n_mma && !warp_failed) {
            produce(produced);
            ++produced;
        }
    }
    if (!failed && issued > 0) {
        bool done = td3tc::mbar_wait(&bar_mma[(issued - 1) & 1], (uint32_t)((issued - 1) >> 1) & 1u,
                                     G_WAIT);
        if (__syncthreads_and(done)) {
            td3tc::fence_after_sync();
            read_out<P, V>(tmem + lane_base + G_D_COL + 64 * ((issued - 1) & 1), prev_live, acc);
        } else {
            failed = true;
        }
    }
    if (failed) {
        if (tid == 0) td3_report(status, 1);
        // drain: the copies of every produced stage not yet consumed and the products
        for (int i = issued; i < produced; ++i)
            td3tc::mbar_wait(&bar_stage[i % G_STAGES], (uint32_t)(i / G_STAGES) & 1u, G_WAIT);
        for (int i = issued - 2 < 0 ? 0 : issued - 2; i < issued; ++i)
            td3tc::mbar_wait(&bar_mma[i & 1], (uint32_t)(i >> 1) & 1u, G_WAIT);
    } else {
        const i64 qp = (i64)tile * G_THREADS + tid;
        const i64 d = qp < n_nodes ? node_at(L, qp) : -1;
        // translations off the operator table: this row's, in the sorted order
        if (jm < j1 && d >= 0) {
            float fv[32];
#pragma unroll
            for (int k = 0; k < 32; ++k) fv[k] = 0.0f;
            for (int e = run_start[jm], e1 = run_start[jm + 1]; e < e1; ++e) {
                unsigned val = vals[e];
                if ((int)(val & 127u) != tid) continue;
                offtable_translation<P>(fv, d, (i64)(val >> 7), order, center, half, hat, C);
                touched = true;
            }
#pragma unroll
            for (int k = 0; k < V; ++k) acc[k] += (double)fv[k];
        }
        if (touched && d >= 0) {
            double hd = half[d], inv_h = 1.0 / hd, ln_h = log(hd), scale = 1.0;
            const double a0r = acc[G_A0_ROW], a0i = acc[G_A0_ROW + 1];
#pragma unroll
            for (int l = 0; l <= P; ++l) {
                if (l < w) {
                    double ur = l ? 0.0 : ln_h * a0r, ui = l ? 0.0 : ln_h * a0i;
                    local_re[d * w + l] += acc[2 * l] * scale + ur;
                    local_im[d * w + l] += acc[2 * l + 1] * scale + ui;
                }
                scale *= inv_h;
            }
        }
    }
    td3tc::fence_before_sync();
    __syncthreads();
    td3tc::fence_after_sync();
    if (warp == 0) td3tc::tmem_free(tmem, G_TMEM_COLS);
}

int bits_for(i64 v) {
    int b = 1;
    while (b < 32 && ((i64)1 << b) <= v) ++b;
    return b;
}

int key_bits_for(int span) { return bits_for((i64)n_keys(span)); }

int fill_levels(const int64_t* levels, int64_t n_levels, int64_t n_nodes, GLevels& L) {
    if (n_levels < 1 || n_levels > G_MAX_LEVELS) return TD3_EINVAL;
    L.n = (int)n_levels;
    for (int i = 0; i <= n_levels; ++i) L.start[i] = levels[i];
    if (L.start[0] != 0 || L.start[n_levels] != n_nodes) return TD3_EINVAL;
    for (int i = n_levels + 1; i <= G_MAX_LEVELS; ++i) L.start[i] = n_nodes;
    return TD3_OK;
}

template <int P, bool SMEM_A>
int launch_grouped(const int* tile_run, const int* run_start, const unsigned* keys,
                   const unsigned* vals, i64 n_nodes, const GLevels& L, const double* center,
                   const double* half, const float2* hat, int order, const float* ops, int span,
                   const double* coeff, double* lre, double* lim, i64* status, cudaStream_t s) {
    GCoef<P> C;
    int w = order + 1;
    for (int k = 0; k <= P; ++k)
        for (int l = 0; l <= P; ++l)
            C.c[k * (P + 1) + l] = (k < w && l < w) ? (float)coeff[k * w + l] : 0.0f;
    // at most two CTAs per SM (each holds G_TMEM_COLS of the 512 tensor-memory columns):
    // at least 80 KB of shared memory per CTA
    constexpr int smem = GShape<P>::bytes(SMEM_A) > 80 * 1024 ? GShape<P>::bytes(SMEM_A) : 80 * 1024;
    auto kernel = k_m2l_grouped<P, SMEM_A>;
    TD3_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    i64 n_tiles = (n_nodes + G_THREADS - 1) / G_THREADS;
    kernel<<<(unsigned)n_tiles, G_THREADS, smem, s>>>(
        tile_run, run_start, keys, vals, n_nodes, L, center, half, hat, order, ops,
        key_bits_for(span), n_keys(span), C, lre, lim, status);
    TD3_CHECK_LAUNCH();
    return TD3_OK;
}

template <bool SMEM_A>
int dispatch_grouped(const int* tile_run, const int* run_start, const unsigned* keys,
                     const unsigned* vals, i64 n_nodes, const GLevels& L, const double* center,
                     const double* half, const float2* hat, int order, const float* ops, int span,
                     const double* coeff, double* lre, double* lim, i64* status, cudaStream_t s) {
    if (order <= 4)
        return launch_grouped<4, SMEM_A>(tile_run, run_start, keys, vals, n_nodes, L, center, half,
                                         hat, order, ops, span, coeff, lre, lim, status, s);
    if (order <= 8)
        return launch_grouped<8, SMEM_A>(tile_run, run_start, keys, vals, n_nodes, L, center, half,
                                         hat, order, ops, span, coeff, lre, lim, status, s);
    if (order <= 12)
        return launch_grouped<12, SMEM_A>(tile_run, run_start, keys, vals, n_nodes, L, center, half,
                                          hat, order, ops, span, coeff, lre, lim, status, s);
    return launch_grouped<14, SMEM_A>(tile_run, run_start, keys, vals, n_nodes, L, center, half,
                                      hat, order, ops, span, coeff, lre, lim, status, s);
}

}  // namespace

extern "C" size_t td3_m2l_operators_size(int span) {
    if (span < 1 || span > G_MAX_SPAN) return 0;
    return (size_t)n_keys(span) * G_B_BYTES;
}

extern "C" int td3_m2l_operators(int order, const double* coeff, int span, float* ops,
                                 void* stream) {
    if (order < 0 || order > TD3_M2L_GROUPED_MAX_ORDER || span < 1 || span > G_MAX_SPAN)
        return TD3_EINVAL;
    i64 threads = (i64)n_keys(span) * 1024;
    k_m2l_operators<<<td3_blocks(threads, 256), 256, 0, td3_stream(stream)>>>(order, coeff, span,
                                                                            ops);
    TD3_CHECK_LAUNCH();
    return TD3_OK;
}

extern "C" size_t td3_m2l_groups_workspace_size(int64_t n_pairs) {
    i64 e = 2 * n_pairs;
    size_t sort = td3_sort_workspace(e), scan = td3_scan_workspace(e);
    return 2 * td3_ws_bytes<unsigned>(e) + 2 * td3_ws_bytes<int>(e) + td3_ws_bytes<int>(1) +
           (sort > scan ? sort : scan);
}

extern "C" int td3_m2l_groups(const int64_t* pairs, int64_t n_pairs, const double* node_center,
                              const double* node_half, const int64_t* node_depth,
                              const int64_t* levels, int64_t n_levels, int64_t n_nodes, int span,
                              uint32_t* keys, uint32_t* values, int32_t* tile_run,
                              int32_t* run_start, void* workspace, size_t workspace_bytes,
                              void* stream) {
    if (n_pairs < 0 || n_nodes < 1 || n_nodes >= ((i64)1 << 25) || span < 1 || span > G_MAX_SPAN)
        return TD3_EINVAL;
    GLevels L;
    TD3_TRY_RC(fill_levels(levels, n_levels, n_nodes, L));
    i64 e = 2 * n_pairs;
    if (e >= 0x7fffffffLL) return TD3_EINVAL;
    i64 n_tiles = (n_nodes + G_THREADS - 1) / G_THREADS;
    int kb = key_bits_for(span);
    int bits = bits_for(n_tiles - 1 > 0 ? n_tiles - 1 : 1) + kb;
    if (bits > 32) return TD3_EINVAL;
    cudaStream_t s = td3_stream(stream);
    if (e == 0) {
        TD3_TRY(cudaMemsetAsync(tile_run, 0, sizeof(int) * (n_tiles + 1), s));
        TD3_TRY(cudaMemsetAsync(run_start, 0, sizeof(int), s));
        return TD3_OK;
    }
    Workspace w(workspace, workspace_bytes);
    unsigned* k1 = w.take<unsigned>(e);
    unsigned* v1 = w.take<unsigned>(e);
    int* flag = w.take<int>(e);
    int* rank = w.take<int>(e);
    int* total = w.take<int>(1);
    if (!total) return TD3_EWORKSPACE;
    // the sort ping-pongs once per 8-bit pass: start where the last pass ends in `keys`
    int passes = (bits + 7) / 8;
    unsigned* k0 = (passes & 1) ? k1 : keys;
    unsigned* v0 = (passes & 1) ? v1 : values;
    unsigned* ka = (passes & 1) ? keys : k1;
    unsigned* va = (passes & 1) ? values : v1;
    k_group_keys<<<td3_blocks(e, 256), 256, 0, s>>>(pairs, n_pairs, node_center, node_half,
                                                    node_depth, L, span, kb, k0, v0);
    TD3_CHECK_LAUNCH();
    unsigned *ko, *vo;
    TD3_TRY_RC(td3_radix_sort_u32(k0, ka, v0, va, e, bits, &ko, &vo, w.base + w.used,
                                  w.size - w.used, s));
    if (ko != keys) return TD3_EINVAL;  // cannot happen: the pass count decides
    k_run_flags<<<td3_blocks(e, 256), 256, 0, s>>>(keys, e, flag);
    TD3_CHECK_LAUNCH();
    TD3_TRY_RC(td3_exclusive_scan_i32(flag, rank, e, total, w.base + w.used, w.size - w.used, s));
    k_run_emit<<<td3_blocks(e + 1, 256), 256, 0, s>>>(keys, flag, rank, total, e, kb, n_tiles,
                                                     tile_run, run_start);
    TD3_CHECK_LAUNCH();
    return TD3_OK;
}

extern "C" int td3_fmm_m2l_grouped(const int32_t* tile_run, const int32_t* run_start,
                                   const uint32_t* keys, const uint32_t* values, int64_t n_nodes,
                                   const int64_t* levels, int64_t n_levels,
                                   const double* node_center, const double* node_half,
                                   const float* hat, int order, const float* ops, int span,
                                   const double* coeff, int smem_operands, double* local_re,
                                   double* local_im, int64_t* status, void* stream) {
    if (n_nodes < 1 || n_nodes >= ((i64)1 << 25) || order < 0 ||
        order > TD3_M2L_GROUPED_MAX_ORDER || span < 1 || span > G_MAX_SPAN || !status)
        return TD3_EINVAL;
    GLevels L;
    TD3_TRY_RC(fill_levels(levels, n_levels, n_nodes, L));
    cudaStream_t s = td3_stream(stream);
    const float2* h = reinterpret_cast<const float2*>(hat);
    if (smem_operands)
        return dispatch_grouped<true>(tile_run, run_start, keys, values, n_nodes, L, node_center,
                                      node_half, h, order, ops, span, coeff, local_re, local_im,
                                      status, s);
    return dispatch_grouped<false>(tile_run, run_start, keys, values, n_nodes, L, node_center,
                                   node_half, h, order, ops, span, coeff, local_re, local_im,
                                   status, s);
}
