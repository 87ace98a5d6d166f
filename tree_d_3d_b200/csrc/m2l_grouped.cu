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

constexpr int G_ROWS = 128;            // destinations per tile; producer threads
constexpr int G_BLOCK = G_ROWS + 32;   // + the MMA-issuing warp
constexpr int G_ASTAGES = 2;           // A stages in tensor memory (hi 32 + lo 32 columns each)
constexpr int G_BSTAGES = 4;           // B stages in shared memory
constexpr int G_BAHEAD = 2;            // a run's B is fetched when the products of run - 2 go
constexpr int G_LAG = 3;               // a run's rows are stored 3 runs after their fetch
constexpr int G_RSTAGES = G_LAG + 1;   // row stages in shared memory
constexpr int G_GROUP = 4;             // runs of one tile summed in one accumulator
constexpr int G_DBUF = 2;              // accumulators of 64 tensor-memory columns
constexpr int G_FIFO = 8;              // groups waiting for their readout (at most 6)
constexpr int G_KRING = 8;             // keys of the runs noted, for the operator copies
constexpr unsigned G_NO_RUN = 0xffffffffu;
constexpr int G_B_BYTES = 8192;        // one key: 64 rows (B_hi, B_lo) x 32 columns of TF32
constexpr int G_RSTRIDE = 144;         // bytes per row in a row stage (odd multiple of 16)
constexpr int G_RSTAGE_BYTES = G_ROWS * G_RSTRIDE;
constexpr int G_LBO = 128;             // bytes between core matrices along K
constexpr int G_SBO = 1024;            // bytes between groups of 8 rows (K = 32)
constexpr int G_D_COL = 0;             // accumulators: tensor-memory columns [0, 128)
constexpr int G_A_COL = G_DBUF * 64;   // A stages: [128, 256)
constexpr int G_TMEM_COLS = 256;       // two CTAs per SM
constexpr int G_OFF_B = 0;
constexpr int G_OFF_ROWS = G_OFF_B + G_BSTAGES * G_B_BYTES;
constexpr int G_OFF_ROWSRC = G_OFF_ROWS + G_RSTAGES * G_RSTAGE_BYTES;  // int[2][128]
constexpr int G_OFF_INFO = G_OFF_ROWSRC + 2 * G_ROWS * 4;               // int[G_ASTAGES]
constexpr int G_OFF_KEYS = G_OFF_INFO + G_ASTAGES * 4;                  // unsigned[G_KRING]
constexpr int G_OFF_FIFO = (G_OFF_KEYS + G_KRING * 4 + 15) & ~15;       // int4[G_FIFO]
// barriers: full, aempty (G_ASTAGES); bfull, bempty (G_BSTAGES); dfull, dempty; drain
constexpr int G_OFF_BARS = G_OFF_FIFO + G_FIFO * 16;
constexpr int G_N_BARS = 2 * G_ASTAGES + 2 * G_BSTAGES + 2 * G_DBUF + 1;
constexpr int G_SMEM = G_OFF_BARS + G_N_BARS * 8 + 16;
static_assert(2 * (G_SMEM + 1024) <= 228 * 1024, "two CTAs per SM");
constexpr int G_FIRST = 1, G_LAST = 2, G_END = 16;  // stage info: bits 2-3 the accumulator
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
    double c[(P + 1) * (P + 1)];
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
    i64 qp = quad_pos(L, d);
    // off the table: a key per destination row past the table's keys, so that each row's
    // off-table translations form one run at the end of its tile
    unsigned key = n_keys(span) + (unsigned)(qp & 127);
    if (dl >= -1 && dl <= 1 && fabs(ux - rx) <= 1e-9 && fabs(uy - ry) <= 1e-9 &&
        fabs(rx) <= span && fabs(ry) <= span)
        key = (unsigned)(((int)(dl + 1) * side + (int)rx + span) * side + (int)ry + span);
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
// The first i in [0, n) with a[i] >= value (n if none), a sorted; every thread of the
// block calls it (a 128-way search: one load and one block barrier per round).
__device__ int block_lower_bound(const int* __restrict__ a, int n, i64 value) {
    int lo = 0, hi = n;
    while (hi > lo) {
        int stride = (hi - lo + 127) / 128;
        int i = lo + (int)threadIdx.x * stride;
        bool below = threadIdx.x < 128 && i < hi && (i64)a[i] < value;
        int nb = __syncthreads_count(below);
        if (nb == 0) break;
        int nhi = lo + nb * stride;
        lo += (nb - 1) * stride + 1;
        hi = nhi < hi ? nhi : hi;
    }
    return lo;
}

// A wait that also gives up when another role of the CTA has raised `abort_flag`.
__device__ __forceinline__ bool wait_or_abort(uint64_t* bar, uint32_t parity,
                                              const volatile int* abort_flag) {
    for (uint32_t i = 0; i < G_WAIT; ++i) {
        if (td3tc::mbar_test(bar, parity)) return true;
        if (*abort_flag) return false;
        if (i > 64) __nanosleep(32);
    }
    return false;
}

// Barrier 1 among the producer warps, returning whether any of them passed `pred`.
__device__ __forceinline__ bool producers_sync_or(bool pred) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 p, %1, 0;\n\t"
        "bar.red.or.pred q, 1, %2, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t}"
        : "=r"(r)
        : "r"((uint32_t)pred), "n"(G_ROWS)
        : "memory");
    return r != 0;
}

// The table's products, a persistent grid of two CTAs per SM over even shares of the
// runs (cut at tile boundaries), warp-specialised:
//   warps 0-3, thread m = row m of every tile (tensor-memory lane m): per run, the
//     translations note their rows in a row table; thread m fetches its row's source
//     (the FP32 scaled moments) by cp.async into its own slot of a row stage and, G_LAG
//     runs later, splits it into TF32 hi + lo (Veltkamp's split on the FP32 pipe: hi
//     keeps 11 significant bits, lo = x - hi exactly) and stores both into the run's A
//     stage in tensor memory (zeros for a row the run leaves out), then arrives on the
//     stage's `full` barrier;
//   warp 4, one thread: per run, waits `full` and `bfull`, issues D = A_hi [B_hi; B_lo]^T
//     (N = 64) and D[:, 0:32] += A_lo B_hi^T (N = 32), K = 32 as four steps of 8, A from
//     tensor memory and B from shared memory, and commits them to the A and B stages'
//     `empty` barriers; it fetches each key's B (8 KB, one bulk copy) G_BAHEAD runs
//     ahead; D accumulates G_GROUP runs of one tile (a fresh D at the group's first run)
//     in one of G_DBUF accumulators, committed to `dfull`;
//   warps 0-3 again: two runs after a group's last run was handed over, its accumulator
//     (FP32 columns 0:32 + 32:64) is added to the row's FP64 sums and released (`dempty`);
//     after a tile's last group the sums go to the locals.
// Sums run in the runs' order: deterministic.  Every wait is bounded; a wait that runs
// out raises the CTA's abort flag and the status word, and the CTA drains its copies and
// products before it releases its tensor memory.
template <int P>
__global__ void __launch_bounds__(G_BLOCK, 2)
k_m2l_grouped(const int* __restrict__ tile_run, const int* __restrict__ run_start,
              const unsigned* __restrict__ keys, const unsigned* __restrict__ vals, int n_tiles,
              i64 n_nodes, GLevels L, const double* __restrict__ half,
              const float2* __restrict__ hat, int order, const float* __restrict__ ops,
              int key_bits, unsigned offtable_key, double* __restrict__ local_re,
              double* __restrict__ local_im, i64* status) {
    extern __shared__ __align__(1024) unsigned char smem[];
    const int tid = threadIdx.x, warp = tid >> 5;
    unsigned char* bstage = smem + G_OFF_B;
    unsigned char* rows = smem + G_OFF_ROWS;
    int* row_src = reinterpret_cast<int*>(smem + G_OFF_ROWSRC);
    int* info = reinterpret_cast<int*>(smem + G_OFF_INFO);
    unsigned* kring = reinterpret_cast<unsigned*>(smem + G_OFF_KEYS);
    int4* fifo = reinterpret_cast<int4*>(smem + G_OFF_FIFO);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + G_OFF_BARS);
    uint64_t* aempty = full + G_ASTAGES;
    uint64_t* bfull = aempty + G_ASTAGES;
    uint64_t* bempty = bfull + G_BSTAGES;
    uint64_t* dfull = bempty + G_BSTAGES;
    uint64_t* dempty = dfull + G_DBUF;
    uint64_t* drain = dempty + G_DBUF;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

    // this CTA's runs [r0, r1)
    const int total = tile_run[n_tiles];
    const i64 share = ((i64)total + gridDim.x - 1) / gridDim.x;
    int t0 = block_lower_bound(tile_run, n_tiles + 1, (i64)blockIdx.x * share);
    int t1 = block_lower_bound(tile_run, n_tiles + 1, (i64)(blockIdx.x + 1) * share);
    t0 = t0 < n_tiles ? t0 : n_tiles;
    t1 = t1 < n_tiles ? t1 : n_tiles;
    const int r0 = tile_run[t0], r1 = tile_run[t1];

    if (tid == 0) {
        for (int s = 0; s < G_ASTAGES; ++s) {
            td3tc::mbar_init(&full[s], G_ROWS);  // the rows' threads, after their stores
            td3tc::mbar_init(&aempty[s], 1);     // the products that read the A stage
        }
        for (int s = 0; s < G_BSTAGES; ++s) {
            td3tc::mbar_init(&bfull[s], 1);   // the B copy's bytes
            td3tc::mbar_init(&bempty[s], 1);  // the products that read the B stage
        }
        for (int b = 0; b < G_DBUF; ++b) {
            td3tc::mbar_init(&dfull[b], 1);
            td3tc::mbar_init(&dempty[b], G_ROWS);
        }
        td3tc::mbar_init(drain, 1);
        *abort_flag = 0;
    }
    for (int i = tid; i < 2 * G_ROWS; i += G_BLOCK) row_src[i] = 0;
    if (warp == 0) td3tc::tmem_alloc(tmem_slot, G_TMEM_COLS);
    td3tc::fence_before_sync();
    __syncthreads();
    td3tc::fence_after_sync();
    const uint32_t tmem = *tmem_slot;

    if (tid < G_ROWS) {
        // ------------------------------------------------ producers and readout
        const int w = order + 1, hw = td3_hat_width(order), chunks = hw / 2;
        const unsigned key_mask = (1u << key_bits) - 1u;
        const uint32_t lane_base = (uint32_t)(32 * warp) << 16;
        unsigned char* my_row = rows + tid * G_RSTRIDE;
        // run data loaded ahead: the starts of runs j .. j + 3, the keys of j .. j + 2
        // (past r1: all ones, an off-table key of no tile) and this thread's entries of
        // runs j and j + 1
        auto start_of = [&](int j) { return run_start[j < r1 ? j : r1]; };
        auto key_of = [&](int j, int start) { return j < r1 ? keys[start] : 0xffffffffu; };
        int j = r0;
        int s0 = start_of(j), s1 = start_of(j + 1), s2 = start_of(j + 2), s3 = start_of(j + 3);
        unsigned k0 = key_of(j, s0), k1 = key_of(j + 1, s1), k2 = key_of(j + 2, s2);
        unsigned v0 = j < r1 && tid < s1 - s0 ? vals[s0 + tid] : 0u;
        unsigned v1 = j + 1 < r1 && tid < s2 - s1 ? vals[s1 + tid] : 0u;

        // FP64 sums of the columns an order up to P uses: bhat_l (re, im) in 2l, 2l + 1,
        // then a_0 (D columns G_A0_ROW, G_A0_ROW + 1)
        constexpr int NV = 2 * (P + 1) + 2;
        double acc[NV];
#pragma unroll
        for (int k = 0; k < NV; ++k) acc[k] = 0.0;
        int qn = 0, qc = 0;  // runs noted (rows fetched), runs consumed (A stored)
        int grp = 0, in_grp = 0, head = 0, tail = 0;
        unsigned live_bits = 0;  // bit i: this row takes part in run qn - 1 - i
        unsigned pend_info = 0;  // byte i: the stage info of run qn - 1 - i
        bool ok = true;

        // the accumulator of group rec.y into the FP64 sums; after a tile's last group,
        // the sums into the locals
        auto readout = [&](int4 rec) {
            const int g = rec.y, buf = g % G_DBUF;
            bool done = td3tc::mbar_wait(&dfull[buf], (uint32_t)(g / G_DBUF) & 1u, G_WAIT);
            done = __all_sync(0xffffffffu, done);
            if (done) {
                td3tc::fence_after_sync();
                // the two column halves (hi and lo products) each added in FP64
#pragma unroll
                for (int half_d = 0; half_d < 2; ++half_d) {
                    float dv[32];
                    td3tc::tmem_load32(tmem + lane_base + G_D_COL + buf * 64 + 32 * half_d, dv);
#pragma unroll
                    for (int k = 0; k < NV; ++k)
                        acc[k] += (double)dv[k < NV - 2 ? k : G_A0_ROW + k - (NV - 2)];
                }
                td3tc::fence_before_sync();
            }
            td3tc::mbar_arrive(&dempty[buf]);
            ok = ok && done;
            if (rec.w) {
                const i64 qp = (i64)rec.z * G_ROWS + tid;
                bool any = false;
#pragma unroll
                for (int k = 0; k < NV; ++k) any |= acc[k] != 0.0;
                if (any && qp < n_nodes) {
                    const i64 d = node_at(L, qp);
                    double* lr = local_re + d * w;
                    double* li = local_im + d * w;
                    // the sums scaled in place: b_l = bhat_l / h^l (+ a_0 ln h for l = 0)
                    double hd = half[d], inv_h = 1.0 / hd, scale = 1.0;
                    acc[0] += log(hd) * acc[NV - 2];
                    acc[1] += log(hd) * acc[NV - 1];
#pragma unroll
                    for (int l = 0; l <= P; ++l) {
                        acc[2 * l] *= scale;
                        acc[2 * l + 1] *= scale;
                        scale *= inv_h;
                    }
                    // four coefficients at a time: their old values loaded together
#pragma unroll
                    for (int l0 = 0; l0 <= P; l0 += 4) {
                        double o_r[4], o_i[4];
#pragma unroll
                        for (int u = 0; u < 4; ++u) {
                            o_r[u] = l0 + u < w ? lr[l0 + u] : 0.0;
                            o_i[u] = l0 + u < w ? li[l0 + u] : 0.0;
                        }
#pragma unroll
                        for (int u = 0; u < 4; ++u) {
                            if (l0 + u < w && l0 + u <= P) {
                                lr[l0 + u] = o_r[u] + acc[2 * (l0 + u)];
                                li[l0 + u] = o_i[u] + acc[2 * (l0 + u) + 1];
                            }
                        }
                    }
                }
#pragma unroll
                for (int k = 0; k < NV; ++k) acc[k] = 0.0;
            }
        };
        // run qc's A stage: this thread's row (G_LAG cp.async groups ago, or all of them
        // in the drain) split into TF32 hi + lo, stored into tensor memory once the
        // products that last read the stage are done
        auto consume = [&](bool drain_all) {
            const int s = qc % G_ASTAGES, back = qn - 1 - qc;
            const bool live = (live_bits >> back) & 1u;
            const unsigned inf = (pend_info >> (8 * back)) & 0xffu;
            if (drain_all) td3tc::cp_async_wait<0>();
            else td3tc::cp_async_wait<G_LAG>();
            const float4* row = reinterpret_cast<const float4*>(my_row + (qc % G_RSTAGES) * G_RSTAGE_BYTES);
            if (qc >= G_ASTAGES)
                ok = td3tc::mbar_wait(&aempty[s], (uint32_t)(qc / G_ASTAGES - 1) & 1u, G_WAIT) && ok;
            td3tc::fence_after_sync();
            const uint32_t a = tmem + lane_base + G_A_COL + 64 * s;
            // hi, then lo (the row read twice from shared memory: fewer live registers)
#pragma unroll
            for (int part = 0; part < 2; ++part) {
                float v[32];
#pragma unroll
                for (int c = 0; c < 8; ++c) {
                    float4 x4 = (live && c < chunks) ? row[c] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                    float x[4] = {x4.x, x4.y, x4.z, x4.w};
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        // Veltkamp: t = (2^13 + 1) x, hi = t - (t - x) has 11 significant bits
                        float t = __fmul_rn(x[u], 8193.0f);
                        float h = __fsub_rn(t, __fsub_rn(t, x[u]));
                        v[4 * c + u] = part ? __fsub_rn(x[u], h) : h;
                    }
                }
                td3tc::tmem_store32(a + 32 * part, v);
            }
            td3tc::tmem_wait_st();
            td3tc::fence_before_sync();
            if (tid == 0) info[s] = (int)inf;
            td3tc::mbar_arrive(&full[s]);
            ++qc;
        };
        // the readouts of groups whose last run was handed over two runs ago
        auto due_readouts = [&]() {
            while (head < tail) {
                int4 rec = fifo[head % G_FIFO];
                if (qc < rec.x + 3) break;
                readout(rec);
                ++head;
            }
        };

        for (; j < r1; ++j) {
            const unsigned key = k0 & key_mask;
            if (key < offtable_key) {
                const int tile = (int)(k0 >> key_bits);
                // note the run's rows, its flags and key, the group's readout record
                if (tid < s1 - s0) row_src[(qn & 1) * G_ROWS + (v0 & 127u)] = (int)(v0 >> 7) + 1;
                const bool first = in_grp == 0;
                const bool last_of_tile =
                    (k1 >> key_bits) != (unsigned)tile || (k1 & key_mask) >= offtable_key;
                const bool last = last_of_tile || in_grp + 1 == G_GROUP;
                const unsigned inf =
                    (first ? G_FIRST : 0u) | (last ? G_LAST : 0u) | ((unsigned)(grp % G_DBUF) << 2);
                if (tid == 0) {
                    kring[qn % G_KRING] = key;
                    if (last) fifo[tail % G_FIFO] = make_int4(qn, grp, tile, last_of_tile ? 1 : 0);
                }
                if (producers_sync_or(!ok)) {  // one decision for the four warps
                    ok = false;
                    break;
                }
                // this thread's row of the run: fetch its source
                const int src1 = row_src[(qn & 1) * G_ROWS + tid];
                row_src[(qn & 1) * G_ROWS + tid] = 0;
                if (src1) {
                    const float2* hrow = hat + (size_t)(src1 - 1) * hw;
                    unsigned char* dst = my_row + (qn % G_RSTAGES) * G_RSTAGE_BYTES;
                    for (int c = 0; c < chunks; ++c) td3tc::cp_async16(dst + 16 * c, hrow + 2 * c);
                }
                td3tc::cp_async_commit();
                live_bits = (live_bits << 1) | (src1 ? 1u : 0u);
                pend_info = (pend_info << 8) | inf;
                if (last) {
                    ++tail;
                    ++grp;
                    in_grp = 0;
                } else {
                    ++in_grp;
                }
                ++qn;
                // the A stage of run qn - 1 - G_LAG
                if (qn > G_LAG) consume(false);
                due_readouts();
            }
            s0 = s1;
            s1 = s2;
            s2 = s3;
            s3 = start_of(j + 4);
            k0 = k1;
            k1 = k2;
            k2 = key_of(j + 3, s2);
            v0 = v1;
            v1 = j + 2 < r1 && tid < s2 - s1 ? vals[s1 + tid] : 0u;
        }
        if (!producers_sync_or(!ok)) {
            // the drain: no operator past the last run, the last runs' A stages, the end
            // marker, the last groups
            if (tid == 0)
                for (int r = qn; r < qn + G_BAHEAD; ++r) kring[r % G_KRING] = G_NO_RUN;
            while (qc < qn) {
                consume(true);
                due_readouts();
            }
            const int s = qn % G_ASTAGES;
            if (qn >= G_ASTAGES)
                ok = td3tc::mbar_wait(&aempty[s], (uint32_t)(qn / G_ASTAGES - 1) & 1u, G_WAIT) && ok;
            if (tid == 0) info[s] = G_END;
            td3tc::mbar_arrive(&full[s]);
            while (head < tail) {
                readout(fifo[head % G_FIFO]);
                ++head;
            }
        } else {
            ok = false;
        }
        td3tc::cp_async_wait<0>();
        if (!ok) {
            *abort_flag = 1;
            td3_report(status, 1);
        }
    } else if (tid == G_ROWS) {
        // ------------------------------------------------ the MMA issuer
        constexpr uint32_t id64 = td3tc::idesc_tf32(G_ROWS, 64);
        constexpr uint32_t id32 = td3tc::idesc_tf32(G_ROWS, 32);
        int q = 0, g = 0, fetched = 0;
        bool ok = true;
        for (;;) {
            const int s = q % G_ASTAGES, bs = q % G_BSTAGES;
            if (!wait_or_abort(&full[s], (uint32_t)(q / G_ASTAGES) & 1u, abort_flag)) {
                ok = false;
                break;
            }
            const int inf = *reinterpret_cast<volatile int*>(&info[s]);
            if (inf & G_END) break;
            // the operators of runs up to q + G_BAHEAD (their keys are noted by now)
            while (ok && fetched <= q + G_BAHEAD) {
                const unsigned key = *reinterpret_cast<volatile unsigned*>(&kring[fetched % G_KRING]);
                if (key == G_NO_RUN) break;
                const int fs = fetched % G_BSTAGES;
                if (fetched >= G_BSTAGES &&
                    !wait_or_abort(&bempty[fs], (uint32_t)(fetched / G_BSTAGES - 1) & 1u, abort_flag)) {
                    ok = false;
                    break;
                }
                td3tc::mbar_arrive_expect_tx(&bfull[fs], G_B_BYTES);
                td3tc::bulk_g2s(bstage + fs * G_B_BYTES, ops + (size_t)key * (G_B_BYTES / 4),
                                G_B_BYTES, &bfull[fs]);
                ++fetched;
            }
            if (!ok || !wait_or_abort(&bfull[bs], (uint32_t)(q / G_BSTAGES) & 1u, abort_flag)) {
                ok = false;
                break;
            }
            const int buf = (inf >> 2) & (G_DBUF - 1);
            if ((inf & G_FIRST) && g >= G_DBUF &&
                !wait_or_abort(&dempty[buf], (uint32_t)(g / G_DBUF - 1) & 1u, abort_flag)) {
                ok = false;
                break;
            }
            td3tc::fence_after_sync();
            const uint32_t bb = td3tc::smem_addr(bstage + bs * G_B_BYTES);
            const uint32_t d = tmem + G_D_COL + buf * 64;
            const uint32_t a = tmem + G_A_COL + 64 * s;
#pragma unroll
            for (int ks = 0; ks < 4; ++ks) {
                uint64_t db = td3tc::smem_desc(bb + 2 * G_LBO * ks, G_LBO, G_SBO);
                td3tc::mma_tf32_ts(d, a + 8 * ks, db, id64, ((inf & G_FIRST) && ks == 0) ? 0u : 1u);
            }
#pragma unroll
            for (int ks = 0; ks < 4; ++ks) {
                uint64_t db = td3tc::smem_desc(bb + 2 * G_LBO * ks, G_LBO, G_SBO);
                td3tc::mma_tf32_ts(d, a + 32 + 8 * ks, db, id32, 1u);
            }
            td3tc::mma_commit(&aempty[s]);
            td3tc::mma_commit(&bempty[bs]);
            if (inf & G_LAST) {
                td3tc::mma_commit(&dfull[buf]);
                ++g;
            }
            ++q;
        }
        // every product issued has completed before the tensor memory is released
        td3tc::mma_commit(drain);
        td3tc::mbar_wait(drain, 0, G_WAIT);
        if (!ok) {
            *abort_flag = 1;
            td3_report(status, 1);
            // the operator copies still in flight (the last use of each stage)
            for (int f = fetched - G_BSTAGES < 0 ? 0 : fetched - G_BSTAGES; f < fetched; ++f)
                td3tc::mbar_wait(&bfull[f % G_BSTAGES], (uint32_t)(f / G_BSTAGES) & 1u, G_WAIT);
        }
    }
    td3tc::fence_before_sync();
    __syncthreads();
    td3tc::fence_after_sync();
    if (warp == 0) td3tc::tmem_free(tmem, G_TMEM_COLS);
}

// The per-translation formula (as k_m2l_mixed) in FP64 for one off-table translation
// into destination d, from the FP32 scaled moments: with ws = h_src / t and wd = h_dst / t,
// a'_k = hat_k ws^k, s_l = sum_k coeff[k, l] a'_k, bhat_0 = a'_0 ln|t / h_dst| - s_0 and
// bhat_l = -(-1)^l s_l wd^l, written to out[2l], out[2l + 1] (l <= P), then a_0 to
// out[2 (P + 1)], out[2 (P + 1) + 1].  FP64 because these translations (large depth
// differences) are few and their sums carry the largest coefficients.
template <int P>
__device__ __forceinline__ void offtable_translation(double* out, i64 d, i64 src, int order,
                                                     const double* __restrict__ center,
                                                     const double* __restrict__ half,
                                                     const float2* __restrict__ hat,
                                                     const GCoef<P>& C) {
    constexpr int W = P + 1;
    const int w = order + 1;
    double tr = center[2 * d] - center[2 * src], ti = center[2 * d + 1] - center[2 * src + 1];
    double t2 = tr * tr + ti * ti, inv = 1.0 / t2, hd = half[d], hs = half[src];
    double wsr = hs * tr * inv, wsi = -hs * ti * inv;
    double wdr = hd * tr * inv, wdi = -hd * ti * inv;
    double lnt = 0.5 * log(t2 / (hd * hd));
    const float2* row = hat + src * td3_hat_width(order);
    double ar[W], ai[W];
    double pr = 1.0, pi = 0.0;
#pragma unroll
    for (int k = 0; k < W; ++k) {
        float2 m = k < w ? row[k] : make_float2(0.0f, 0.0f);
        ar[k] = (double)m.x * pr - (double)m.y * pi;
        ai[k] = (double)m.x * pi + (double)m.y * pr;
        double nr = pr * wsr - pi * wsi;
        pi = pr * wsi + pi * wsr;
        pr = nr;
    }
    double qr = 1.0, qi = 0.0;
#pragma unroll
    for (int l = 0; l < W; ++l) {
        double sr = 0.0, si = 0.0;
#pragma unroll
        for (int k = 0; k < W; ++k) {
            sr += C.c[k * W + l] * ar[k];
            si += C.c[k * W + l] * ai[k];
        }
        if (l == 0) {
            out[0] = ar[0] * lnt - sr;
            out[1] = ai[0] * lnt - si;
        } else {
            double sign = (l & 1) ? 1.0 : -1.0;
            out[2 * l] = l < w ? sign * (sr * qr - si * qi) : 0.0;
            out[2 * l + 1] = l < w ? sign * (sr * qi + si * qr) : 0.0;
        }
        double nr = qr * wdr - qi * wdi;
        qi = qr * wdi + qi * wdr;
        qr = nr;
    }
    out[2 * W] = ar[0];
    out[2 * W + 1] = ai[0];
}

// The translations off the operator table, a CTA per tile (tiles without any return at
// once): one run per destination row after the tile's table runs.  Thread t evaluates
// entry t of each chunk of 128 into shared scratch, then each row's thread adds its own
// entries, in order, in FP64, and adds the sums to the locals (after the table's
// products: deterministic).
template <int P>
__global__ void __launch_bounds__(G_ROWS)
k_m2l_offtable(const int* __restrict__ tile_run, const int* __restrict__ run_start,
               const unsigned* __restrict__ keys, const unsigned* __restrict__ vals,
               i64 n_nodes, GLevels L, const double* __restrict__ center,
               const double* __restrict__ half, const float2* __restrict__ hat, int order,
               int key_bits, unsigned offtable_key, const GCoef<P> C,
               double* __restrict__ local_re, double* __restrict__ local_im) {
    constexpr int NV = 2 * (P + 1) + 2;  // bhat_l (re, im), then a_0
    constexpr int NS = NV + 1;           // doubles per scratch slot (odd: no bank conflicts)
    extern __shared__ double off_scratch[];
    const int tid = threadIdx.x, tile = blockIdx.x;
    const int j0 = tile_run[tile], j1 = tile_run[tile + 1];
    if (j0 == j1) return;
    const unsigned key_mask = (1u << key_bits) - 1u;
    const int n_off = __syncthreads_count(
        tid < j1 - j0 && (keys[run_start[j1 - 1 - tid]] & key_mask) >= offtable_key);
    if (n_off == 0) return;
    const int jm = j1 - n_off;
    int* own = reinterpret_cast<int*>(off_scratch + G_ROWS * NS);  // 2 x 128
    own[tid] = 0;
    own[G_ROWS + tid] = 0;
    __syncthreads();
    if (tid < n_off) {
        int r = jm + tid, row = (int)((keys[run_start[r]] & key_mask) - offtable_key);
        own[row] = run_start[r];
        own[G_ROWS + row] = run_start[r + 1];
    }
    __syncthreads();
    const int my0 = own[tid], my1 = own[G_ROWS + tid];
    double acc[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) acc[k] = 0.0;
    const int e0 = run_start[jm], e1 = run_start[j1];
    for (int base = e0; base < e1; base += G_ROWS) {
        if (base + tid < e1) {
            unsigned val = vals[base + tid];
            i64 de = node_at(L, (i64)tile * G_ROWS + (val & 127u));
            offtable_translation<P>(off_scratch + tid * NS, de, (i64)(val >> 7), order, center,
                                    half, hat, C);
        }
        __syncthreads();
        const int a = my0 > base ? my0 : base;
        const int b = my1 < base + G_ROWS ? my1 : base + G_ROWS;
        for (int x = a; x < b; ++x) {
            const double* f = off_scratch + (x - base) * NS;
#pragma unroll
            for (int k = 0; k < NV; ++k) acc[k] += f[k];
        }
        __syncthreads();
    }
    const i64 qp = (i64)tile * G_ROWS + tid;
    if (my1 > my0 && qp < n_nodes) {
        const int w = order + 1;
        const i64 d = node_at(L, qp);
        double hd = half[d], inv_h = 1.0 / hd, ln_h = log(hd), scale = 1.0;
#pragma unroll
        for (int l = 0; l <= P; ++l) {
            if (l < w) {
                double ur = l ? 0.0 : ln_h * acc[NV - 2];
                double ui = l ? 0.0 : ln_h * acc[NV - 1];
                local_re[d * w + l] += acc[2 * l] * scale + ur;
                local_im[d * w + l] += acc[2 * l + 1] * scale + ui;
            }
            scale *= inv_h;
        }
    }
}

int bits_for(i64 v) {
    int b = 1;
    while (b < 32 && ((i64)1 << b) <= v) ++b;
    return b;
}

int key_bits_for(int span) { return bits_for((i64)n_keys(span) + G_ROWS - 1); }

int fill_levels(const int64_t* levels, int64_t n_levels, int64_t n_nodes, GLevels& L) {
    if (n_levels < 1 || n_levels > G_MAX_LEVELS) return TD3_EINVAL;
    L.n = (int)n_levels;
    for (int i = 0; i <= n_levels; ++i) L.start[i] = levels[i];
    if (L.start[0] != 0 || L.start[n_levels] != n_nodes) return TD3_EINVAL;
    for (int i = n_levels + 1; i <= G_MAX_LEVELS; ++i) L.start[i] = n_nodes;
    return TD3_OK;
}

template <int P>
int launch_grouped(const int* tile_run, const int* run_start, const unsigned* keys,
                   const unsigned* vals, i64 n_nodes, const GLevels& L, const double* center,
                   const double* half, const float2* hat, int order,
                   const float* ops, int span, const double* coeff, double* lre, double* lim,
                   i64* status, cudaStream_t s) {
    const i64 n_tiles = (n_nodes + G_ROWS - 1) / G_ROWS;
    const int kb = key_bits_for(span);
    int dev = 0, n_sm = 0;
    TD3_TRY(cudaGetDevice(&dev));
    TD3_TRY(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev));
    auto grouped = k_m2l_grouped<P>;
    TD3_TRY(cudaFuncSetAttribute(grouped, cudaFuncAttributeMaxDynamicSharedMemorySize, G_SMEM));
    const i64 grid = n_tiles < 2 * n_sm ? n_tiles : 2 * n_sm;  // two CTAs per SM
    grouped<<<(unsigned)grid, G_BLOCK, G_SMEM, s>>>(tile_run, run_start, keys, vals, (int)n_tiles,
                                                    n_nodes, L, half, hat, order, ops, kb,
                                                    n_keys(span), lre, lim, status);
    TD3_CHECK_LAUNCH();
    GCoef<P> C;
    int w = order + 1;
    for (int k = 0; k <= P; ++k)
        for (int l = 0; l <= P; ++l)
            C.c[k * (P + 1) + l] = (k < w && l < w) ? coeff[k * w + l] : 0.0;
    constexpr int off_smem = G_ROWS * (2 * (P + 1) + 3) * 8 + 2 * G_ROWS * 4;
    k_m2l_offtable<P><<<(unsigned)n_tiles, G_ROWS, off_smem, s>>>(
        tile_run, run_start, keys, vals, n_nodes, L, center, half, hat, order, kb, n_keys(span), C,
        lre, lim);
    TD3_CHECK_LAUNCH();
    return TD3_OK;
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
    i64 n_tiles = (n_nodes + G_ROWS - 1) / G_ROWS;
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
                                   const float* hat, int order, const float* ops,
                                   int span, const double* coeff, double* local_re,
                                   double* local_im, int64_t* status, void* stream) {
    if (n_nodes < 1 || n_nodes >= ((i64)1 << 25) || order < 0 ||
        order > TD3_M2L_GROUPED_MAX_ORDER || span < 1 || span > G_MAX_SPAN || !status)
        return TD3_EINVAL;
    GLevels L;
    TD3_TRY_RC(fill_levels(levels, n_levels, n_nodes, L));
    cudaStream_t s = td3_stream(stream);
    const float2* h = reinterpret_cast<const float2*>(hat);
    if (order <= 4)
        return launch_grouped<4>(tile_run, run_start, keys, values, n_nodes, L, node_center,
                                 node_half, h, order, ops, span, coeff, local_re, local_im,
                                 status, s);
    if (order <= 8)
        return launch_grouped<8>(tile_run, run_start, keys, values, n_nodes, L, node_center,
                                 node_half, h, order, ops, span, coeff, local_re, local_im,
                                 status, s);
    if (order <= 12)
        return launch_grouped<12>(tile_run, run_start, keys, values, n_nodes, L, node_center,
                                  node_half, h, order, ops, span, coeff, local_re, local_im,
                                  status, s);
    return launch_grouped<14>(tile_run, run_start, keys, values, n_nodes, L, node_center,
                              node_half, h, order, ops, span, coeff, local_re, local_im,
                              status, s);
}
