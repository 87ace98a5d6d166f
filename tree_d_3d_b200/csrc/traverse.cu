// Interaction lists of the FMM:
//   fmm_traverse   mutual dual-tree traversal from (root, root), generation by
//                  generation (K/fmm_traverse/fmm_traverse_pyccel.py:15-106, driven by
//                  FlatQuadtree._traverse, ft:1318-1358);
//   dual_traverse  one-way traversal of a target tree against a source tree
//                  (K/dual_traverse/dual_traverse_pyccel.py:14-86);
//   pair_csr       pair lists as rows by node (K/pair_csr/pair_csr_pyccel.py:12-45).
//
// A generation classifies every frontier pair (M2L, P2P, its 4 or 10 child pairs, or
// dropped), an exclusive scan of the per-pair counts gives each output its slot, and a
// second pass writes them: the lists come out in the reference's serial order.  The
// frontier sizes stay on the device; the host looks at them every few generations.  The
// predicates use exactly rounded operations (this file is compiled with --fmad=false).
#include "common.cuh"

namespace {

constexpr int TRAV_THREADS = 256;

struct Pair {
    i64 a, b;
};

// A frontier pair: node indices fit 32 bits (the entry points check the node counts).
struct __align__(8) FPair {
    int a, b;
};

enum : int { ACT_NONE = 0, ACT_M2L = 1, ACT_P2P = 2, ACT_SELF = 3, ACT_SPLIT_A = 4, ACT_SPLIT_B = 5 };

// A node as the traversal reads it: one 32-byte record (one memory sector) instead of
// five arrays.  child is the first child (-1 for a leaf), filled is 0 for an empty cell.
struct __align__(32) NodeRec {
    double cx, cy, half;
    int child, filled;
};

__global__ void k_node_records(i64 count, const double* __restrict__ center,
                               const double* __restrict__ half, const i64* __restrict__ start,
                               const i64* __restrict__ end, const i64* __restrict__ child,
                               NodeRec* __restrict__ rec) {
    td3_chain_wait();
    td3_chain_release();
    i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    rec[i] = NodeRec{center[2 * i], center[2 * i + 1], half[i], (int)child[i],
                     end[i] != start[i] ? 1 : 0};
}

// The decision of the mutual traversal for pair (a, b) (fmm_traverse_pyccel.py:48-106).
__device__ __forceinline__ int classify_mutual(i64 a, i64 b, const NodeRec* __restrict__ rec,
                                               double theta) {
    NodeRec ra = rec[a], rb = rec[b];
    if (!ra.filled || !rb.filled) return ACT_NONE;
    bool leaf_a = ra.child < 0, leaf_b = rb.child < 0;
    if (a == b) return leaf_a ? ACT_P2P : ACT_SELF;
    double dx = xsub(ra.cx, rb.cx);
    double dy = xsub(ra.cy, rb.cy);
    double distance = xsqrt(xnorm2(dx, dy));
    double radii = xmul(TD3_ROOT2, xadd(ra.half, rb.half));
    if (radii < xmul(theta, distance)) return ACT_M2L;
    if (leaf_a && leaf_b) return ACT_P2P;
    if (leaf_b || (!leaf_a && ra.half >= rb.half)) return ACT_SPLIT_A;
    return ACT_SPLIT_B;
}

// counts: a = m2l | (p2p << 32), b = next-frontier pairs
__device__ __forceinline__ td3_i64x2 action_counts(int act) {
    switch (act) {
        case ACT_M2L: return td3_i64x2(1, 0);
        case ACT_P2P: return td3_i64x2((i64)1 << 32, 0);
        case ACT_SELF: return td3_i64x2(0, 10);
        case ACT_SPLIT_A:
        case ACT_SPLIT_B: return td3_i64x2(0, 4);
        default: return td3_i64x2(0, 0);
    }
}

// The one-way decision for (target cell a, source cell b) (dual_traverse_pyccel.py:46-86).
__device__ __forceinline__ int classify_dual(i64 a, i64 b, const NodeRec* __restrict__ t_rec,
                                             const NodeRec* __restrict__ s_rec, double theta) {
    NodeRec ra = t_rec[a], rb = s_rec[b];
    if (!ra.filled || !rb.filled) return ACT_NONE;
    double dx = xsub(ra.cx, rb.cx);
    double dy = xsub(ra.cy, rb.cy);
    if (xmul(TD3_ROOT2, xadd(ra.half, rb.half)) < xmul(theta, xsqrt(xnorm2(dx, dy))))
        return ACT_M2L;
    bool leaf_a = ra.child < 0, leaf_b = rb.child < 0;
    if (leaf_a && leaf_b) return ACT_P2P;
    if (leaf_b || (!leaf_a && ra.half >= rb.half)) return ACT_SPLIT_A;
    return ACT_SPLIT_B;
}

// ------------------------------------------------------------------ generations
// A generation is three launches of fixed size that read the frontier size from device
// memory: classify (action per pair, counts per tile of GEN_TILE pairs), an exclusive
// scan of the tile counts (one block; it also checks the buffers and advances the
// totals), and emit (per tile, block scans of the pairs' counts in frontier order give
// every output its slot).  The host reads the state once per GEN_BATCH generations.
constexpr int GEN_ITEMS = 8;
constexpr int GEN_TILE = TRAV_THREADS * GEN_ITEMS;
constexpr int GEN_BATCH = 8;

struct TravState {
    i64 nf[2];          // frontier size of even / odd generations
    i64 emit_nf;        // frontier size the current emit pass writes (0 after overflow)
    i64 n_m2l, n_p2p;   // pairs listed so far
    i64 base_m2l, base_p2p;
    i64 overflow;       // a list or the next frontier outgrew its buffer
    i64 need_m2l, need_p2p, need_frontier;
    unsigned long long arrived;  // classify blocks done in the current generation
};

template <bool DUAL>
__device__ __forceinline__ int classify_pair(const NodeRec* t, const NodeRec* s, double theta,
                                             FPair pr) {
    if (DUAL) return classify_dual(pr.a, pr.b, t, s, theta);
    return classify_mutual(pr.a, pr.b, t, theta);
}

__device__ __forceinline__ td3_i64x2 warp_inclusive_x2(td3_i64x2 v, int lane) {
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        long long a = __shfl_up_sync(0xffffffffu, (long long)v.a, d);
        long long b = __shfl_up_sync(0xffffffffu, (long long)v.b, d);
        if (lane >= d) {
            v.a += a;
            v.b += b;
        }
    }
    return v;
}

// Exclusive scan over the block (blockDim.x a multiple of 32, at most 1024 threads).
__device__ __forceinline__ td3_i64x2 block_exclusive_x2(td3_i64x2 v, td3_i64x2* total) {
    __shared__ td3_i64x2 sums[32];
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    td3_i64x2 inc = warp_inclusive_x2(v, lane);
    if (lane == 31) sums[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        td3_i64x2 x = lane < nw ? sums[lane] : td3_i64x2(0);
        x = warp_inclusive_x2(x, lane);
        if (lane < nw) sums[lane] = x;
    }
    __syncthreads();
    td3_i64x2 off = warp ? sums[warp - 1] : td3_i64x2(0);
    *total = sums[nw - 1];
    __syncthreads();
    return off + inc - v;
}

__global__ void k_gen_init(TravState* st, FPair* frontier) {
    td3_chain_wait();
    td3_chain_release();
    st->nf[0] = 1;
    st->nf[1] = 0;
    st->emit_nf = 0;
    st->n_m2l = st->n_p2p = st->base_m2l = st->base_p2p = 0;
    st->overflow = st->need_m2l = st->need_p2p = st->need_frontier = 0;
    st->arrived = 0;
    frontier[0] = FPair{0, 0};
}

template <bool DUAL>
__global__ void __launch_bounds__(TRAV_THREADS)
k_gen_classify(const FPair* __restrict__ frontier, TravState* st, int parity,
               const NodeRec* __restrict__ t, const NodeRec* __restrict__ s, double theta,
               signed char* __restrict__ action, td3_i64x2* __restrict__ tile_sum,
               i64 m2l_capacity, i64 p2p_capacity, i64 frontier_capacity) {
    __shared__ bool last;
    td3_chain_wait();
    td3_chain_release();
    i64 nf = st->nf[parity];
    i64 tiles = (nf + GEN_TILE - 1) / GEN_TILE;
    for (i64 tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        td3_i64x2 sum(0);
#pragma unroll
        for (int i = 0; i < GEN_ITEMS; ++i) {
            i64 k = tile * GEN_TILE + i * TRAV_THREADS + threadIdx.x;
            if (k < nf) {
                int act = classify_pair<DUAL>(t, s, theta, frontier[k]);
                action[k] = (signed char)act;
                sum += action_counts(act);
            }
        }
        td3_i64x2 total;
        block_exclusive_x2(sum, &total);
        if (threadIdx.x == 0) tile_sum[tile] = total;
    }
    // The last block to finish scans the tile sums (no block waits: the others leave).
    if (threadIdx.x == 0) {
        __threadfence();  // this block's tile sums before its arrival
        last = atomicAdd(&st->arrived, 1ull) == (unsigned long long)gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    td3_i64x2 carry(0);
    for (i64 c = 0; c < tiles; c += blockDim.x) {
        i64 tile = c + threadIdx.x;
        td3_i64x2 v(0);
        if (tile < tiles) {
            v.a = __ldcg(reinterpret_cast<const long long*>(&tile_sum[tile].a));
            v.b = __ldcg(reinterpret_cast<const long long*>(&tile_sum[tile].b));
        }
        td3_i64x2 total;
        td3_i64x2 ex = block_exclusive_x2(v, &total);
        if (tile < tiles) tile_sum[tile] = carry + ex;
        carry += total;
    }
    if (threadIdx.x == 0) {
        st->arrived = 0;
        i64 add_m2l = carry.a & 0xffffffffLL, add_p2p = carry.a >> 32, nn = carry.b;
        st->base_m2l = st->n_m2l;
        st->base_p2p = st->n_p2p;
        if (st->n_m2l + add_m2l > m2l_capacity || st->n_p2p + add_p2p > p2p_capacity ||
            nn > frontier_capacity) {
            st->overflow = 1;
            st->need_m2l = st->n_m2l + add_m2l;
            st->need_p2p = st->n_p2p + add_p2p;
            st->need_frontier = nn;
            st->emit_nf = 0;
            st->nf[parity ^ 1] = 0;
        } else {
            st->n_m2l += add_m2l;
            st->n_p2p += add_p2p;
            st->emit_nf = nf;
            st->nf[parity ^ 1] = nn;
        }
    }
}

// Emit: a warp takes 32 * GEN_ITEMS consecutive pairs of the tile (round r, lane l:
// pair warp_base + 32 r + l); the warps' totals are scanned once per tile, then each
// round's slots come from a warp scan, in frontier order.
template <bool DUAL>
__global__ void __launch_bounds__(TRAV_THREADS)
k_gen_emit(const FPair* __restrict__ frontier, const TravState* st,
           const signed char* __restrict__ action, const td3_i64x2* __restrict__ tile_off,
           const NodeRec* __restrict__ t_rec, const NodeRec* __restrict__ s_rec,
           Pair* __restrict__ m2l, Pair* __restrict__ p2p, FPair* __restrict__ next) {
    __shared__ td3_i64x2 warp_total[TRAV_THREADS / 32];
    td3_chain_wait();
    td3_chain_release();
    int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    i64 nf = st->emit_nf;
    i64 base_m2l = st->base_m2l, base_p2p = st->base_p2p;
    i64 tiles = (nf + GEN_TILE - 1) / GEN_TILE;
    for (i64 tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        i64 first = tile * GEN_TILE + (i64)wib * 32 * GEN_ITEMS;
        int act[GEN_ITEMS];
        td3_i64x2 mine(0);
#pragma unroll
        for (int r = 0; r < GEN_ITEMS; ++r) {
            i64 k = first + r * 32 + lane;
            act[r] = k < nf ? action[k] : ACT_NONE;
            mine += action_counts(act[r]);
        }
        td3_i64x2 wsum = warp_inclusive_x2(mine, lane);
        __syncthreads();  // the previous tile's readers are done with warp_total
        if (lane == 31) warp_total[wib] = wsum;
        __syncthreads();
        td3_i64x2 carry = tile_off[tile];
        for (int w = 0; w < wib; ++w) carry += warp_total[w];
#pragma unroll
        for (int r = 0; r < GEN_ITEMS; ++r) {
            td3_i64x2 c = action_counts(act[r]);
            td3_i64x2 inc = warp_inclusive_x2(c, lane);
            td3_i64x2 off = carry + inc - c;
            long long ta = __shfl_sync(0xffffffffu, (long long)inc.a, 31);
            long long tb = __shfl_sync(0xffffffffu, (long long)inc.b, 31);
            carry += td3_i64x2(ta, tb);
            if (act[r] == ACT_NONE) continue;
            FPair pr = frontier[first + r * 32 + lane];
            switch (act[r]) {
                case ACT_M2L: m2l[base_m2l + (off.a & 0xffffffffLL)] = Pair{pr.a, pr.b}; break;
                case ACT_P2P: p2p[base_p2p + (off.a >> 32)] = Pair{pr.a, pr.b}; break;
                case ACT_SELF: {
                    int f = t_rec[pr.a].child;
                    i64 j = off.b;
                    for (int c1 = 0; c1 < 4; ++c1)
                        for (int d = c1; d < 4; ++d) next[j++] = FPair{f + c1, f + d};
                    break;
                }
                case ACT_SPLIT_A: {
                    int f = t_rec[pr.a].child;
                    for (int c1 = 0; c1 < 4; ++c1) next[off.b + c1] = FPair{f + c1, pr.b};
                    break;
                }
                default: {
                    int f = (DUAL ? s_rec : t_rec)[pr.b].child;
                    for (int c1 = 0; c1 < 4; ++c1) next[off.b + c1] = FPair{pr.a, f + c1};
                    break;
                }
            }
        }
    }
}

struct TraverseBuffers {
    FPair* frontier[2];
    signed char* action;
    td3_i64x2* tile_sum;
    TravState* state;
    NodeRec* rec[2];  // target (and source) tree records
};

i64 gen_tiles(i64 frontier_cap) { return (frontier_cap + GEN_TILE - 1) / GEN_TILE; }

size_t traverse_workspace(i64 frontier_cap, i64 n_records) {
    return 2 * td3_ws_bytes<FPair>(frontier_cap) + td3_ws_bytes<signed char>(frontier_cap) +
           td3_ws_bytes<td3_i64x2>(gen_tiles(frontier_cap)) + td3_ws_bytes<TravState>(1) +
           td3_ws_bytes<NodeRec>(n_records) + 512;
}

bool take_traverse(Workspace& w, i64 frontier_cap, i64 n_t, i64 n_s, TraverseBuffers& b) {
    b.frontier[0] = w.take<FPair>(frontier_cap);
    b.frontier[1] = w.take<FPair>(frontier_cap);
    b.action = w.take<signed char>(frontier_cap);
    b.tile_sum = w.take<td3_i64x2>(gen_tiles(frontier_cap));
    b.state = w.take<TravState>(1);
    b.rec[0] = w.take<NodeRec>(n_t);
    b.rec[1] = n_s ? w.take<NodeRec>(n_s) : b.rec[0];
    return b.rec[1] != nullptr;
}

int launch_records(i64 count, const double* center, const double* half, const i64* start,
                    const i64* end, const i64* child, NodeRec* rec, cudaStream_t stream) {
    TD3_TRY(td3_launch_chained(k_node_records, td3_blocks(count, 256), 256, 0, stream, count,
                               center, half, start, end, child, rec));
    return TD3_OK;
}

// The generations from (root, root) until the frontier is empty; sizes as the entry
// points document them.
template <bool DUAL>
int run_generations(const NodeRec* t, const NodeRec* s, double theta, Pair* m2l,
                    i64 m2l_capacity, Pair* p2p, i64 p2p_capacity, i64 frontier_capacity,
                    int64_t* sizes, const TraverseBuffers& b, cudaStream_t stream) {
    i64 tiles = gen_tiles(frontier_capacity);
    unsigned grid = (unsigned)(tiles < 148 * 4 ? tiles : 148 * 4);
    TD3_TRY(td3_launch_chained(k_gen_init, 1, 1, 0, stream, b.state, b.frontier[0]));
    TD3_CHECK_LAUNCH();
    sizes[0] = sizes[1] = sizes[2] = sizes[3] = 0;
    for (int gen = 0;;) {
        for (int k = 0; k < GEN_BATCH; ++k, ++gen) {
            int parity = gen & 1;
            TD3_TRY(td3_launch_chained(k_gen_classify<DUAL>, grid, TRAV_THREADS, 0, stream,
                                       (const FPair*)b.frontier[parity], b.state, parity, t, s,
                                       theta, b.action, b.tile_sum, m2l_capacity, p2p_capacity,
                                       frontier_capacity));
            TD3_TRY(td3_launch_chained(k_gen_emit<DUAL>, grid, TRAV_THREADS, 0, stream,
                                       (const FPair*)b.frontier[parity], (const TravState*)b.state,
                                       (const signed char*)b.action,
                                       (const td3_i64x2*)b.tile_sum, t, s, m2l, p2p,
                                       b.frontier[parity ^ 1]));
            TD3_CHECK_LAUNCH();
        }
        TravState h;
        TD3_TRY(cudaMemcpyAsync(&h, b.state, sizeof(h), cudaMemcpyDeviceToHost, stream));
        TD3_TRY(cudaStreamSynchronize(stream));
        if (h.overflow) {
            sizes[0] = h.need_m2l;
            sizes[1] = h.need_p2p;
            sizes[2] = h.need_frontier;
            sizes[3] = -1;
            return TD3_ENEEDMORE;
        }
        if (h.nf[gen & 1] == 0) {
            sizes[0] = h.n_m2l;
            sizes[1] = h.n_p2p;
            return TD3_OK;
        }
    }
}

// ------------------------------------------------------------------ pair CSR
__global__ void k_csr_keys(const Pair* __restrict__ pairs, i64 count, int mutual, unsigned invalid,
                           unsigned* __restrict__ keys, unsigned* __restrict__ vals) {
    td3_chain_wait();
    td3_chain_release();
    i64 p = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= count) return;
    Pair pr = pairs[p];
    if (mutual) {
        keys[2 * p] = (unsigned)pr.a;
        vals[2 * p] = (unsigned)pr.b;
        if (pr.a != pr.b) {
            keys[2 * p + 1] = (unsigned)pr.b;
            vals[2 * p + 1] = (unsigned)pr.a;
        } else {
            keys[2 * p + 1] = invalid;
            vals[2 * p + 1] = 0;
        }
    } else {
        keys[p] = (unsigned)pr.a;
        vals[p] = (unsigned)pr.b;
    }
}

// The CSR from the sorted entries, one thread per position j in [0, e]: partners (int64)
// and, when asked, the row of every entry (int32); and row_start[d] = the first sorted
// position with key >= d (keys sorted, the invalid key n_nodes last), position j setting
// the rows between its predecessor's key and its own.
__global__ void k_csr_out(const unsigned* __restrict__ vals, const unsigned* __restrict__ keys,
                          i64 e, i64 n_nodes, i64* __restrict__ row_start,
                          i64* __restrict__ partners, int* __restrict__ entry_row) {
    td3_chain_wait();
    td3_chain_release();
    i64 j = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (j > e) return;
    i64 prev = j == 0 ? -1 : (i64)keys[j - 1];
    i64 cur = n_nodes;
    if (j < e) {
        unsigned key = keys[j];
        partners[j] = vals[j];
        if (entry_row) entry_row[j] = (int)key;
        cur = (i64)key < n_nodes ? (i64)key : n_nodes;
    }
    for (i64 d = prev + 1; d <= cur; ++d) row_start[d] = j;
}

int bits_for(i64 v) {
    int b = 1;
    while (b < 32 && ((i64)1 << b) <= v) ++b;
    return b;
}

}  // namespace

extern "C" size_t td3_fmm_traverse_workspace_size(int64_t frontier_capacity, int64_t n_nodes) {
    return traverse_workspace(frontier_capacity, n_nodes);
}

extern "C" int td3_fmm_traverse(const double* node_center, const double* node_half,
                                const int64_t* node_start, const int64_t* node_end,
                                const int64_t* node_child, int64_t n_nodes, double theta,
                                int64_t* m2l, int64_t m2l_capacity, int64_t* p2p,
                                int64_t p2p_capacity, int64_t frontier_capacity, int64_t* sizes,
                                void* workspace, size_t workspace_bytes, void* stream) {
    if (frontier_capacity < 1 || m2l_capacity < 0 || p2p_capacity < 0) return TD3_EINVAL;
    if (n_nodes < 1 || n_nodes > 0x7fffffffLL) return TD3_EINVAL;
    Workspace w(workspace, workspace_bytes);
    TraverseBuffers b;
    if (!take_traverse(w, frontier_capacity, n_nodes, 0, b)) return TD3_EWORKSPACE;
    cudaStream_t s = td3_stream(stream);
    TD3_TRY_RC(launch_records(n_nodes, node_center, node_half, node_start, node_end, node_child,
                              b.rec[0], s));
    return run_generations<false>(b.rec[0], b.rec[0], theta, reinterpret_cast<Pair*>(m2l),
                                  m2l_capacity, reinterpret_cast<Pair*>(p2p), p2p_capacity,
                                  frontier_capacity, sizes, b, s);
}

extern "C" int td3_dual_traverse(const double* t_center, const double* t_half,
                                 const int64_t* t_start, const int64_t* t_end,
                                 const int64_t* t_child, int64_t t_nodes, const double* s_center,
                                 const double* s_half, const int64_t* s_start,
                                 const int64_t* s_end, const int64_t* s_child, int64_t s_nodes,
                                 double theta, int64_t* m2l, int64_t m2l_capacity, int64_t* p2p,
                                 int64_t p2p_capacity, int64_t frontier_capacity, int64_t* sizes,
                                 void* workspace, size_t workspace_bytes, void* stream) {
    if (frontier_capacity < 1 || m2l_capacity < 0 || p2p_capacity < 0) return TD3_EINVAL;
    if (t_nodes < 1 || s_nodes < 1 || t_nodes > 0x7fffffffLL || s_nodes > 0x7fffffffLL)
        return TD3_EINVAL;
    Workspace w(workspace, workspace_bytes);
    TraverseBuffers b;
    if (!take_traverse(w, frontier_capacity, t_nodes, s_nodes, b)) return TD3_EWORKSPACE;
    cudaStream_t s = td3_stream(stream);
    TD3_TRY_RC(launch_records(t_nodes, t_center, t_half, t_start, t_end, t_child, b.rec[0], s));
    TD3_TRY_RC(launch_records(s_nodes, s_center, s_half, s_start, s_end, s_child, b.rec[1], s));
    return run_generations<true>(b.rec[0], b.rec[1], theta, reinterpret_cast<Pair*>(m2l),
                                 m2l_capacity, reinterpret_cast<Pair*>(p2p), p2p_capacity,
                                 frontier_capacity, sizes, b, s);
}

extern "C" size_t td3_pair_csr_workspace_size(int64_t count, int mutual, int64_t n_nodes) {
    i64 e = mutual ? 2 * count : count;
    size_t sort = td3_sort_workspace(e), scan = td3_scan_workspace(n_nodes + 1);
    return 4 * td3_ws_bytes<unsigned>(e) + (sort > scan ? sort : scan);
}

extern "C" int td3_pair_csr(const int64_t* pairs, int64_t count, int mutual, int64_t n_nodes,
                            int64_t* row_start, int64_t* partners, int32_t* entry_row,
                            void* workspace, size_t workspace_bytes, void* stream) {
    if (count < 0 || n_nodes < 1 || n_nodes >= 0x7fffffffLL) return TD3_EINVAL;
    cudaStream_t s = td3_stream(stream);
    if (count == 0) {
        TD3_TRY(cudaMemsetAsync(row_start, 0, sizeof(i64) * (n_nodes + 1), s));
        return TD3_OK;
    }
    i64 e = mutual ? 2 * count : count;
    Workspace w(workspace, workspace_bytes);
    unsigned* k0 = w.take<unsigned>(e);
    unsigned* k1 = w.take<unsigned>(e);
    unsigned* v0 = w.take<unsigned>(e);
    unsigned* v1 = w.take<unsigned>(e);
    if (!v1) return TD3_EWORKSPACE;
    TD3_TRY(td3_launch_chained(k_csr_keys, td3_blocks(count, 256), 256, 0, s,
                               reinterpret_cast<const Pair*>(pairs), count, mutual,
                               (unsigned)n_nodes, k0, v0));
    TD3_CHECK_LAUNCH();
    unsigned *ko, *vo;
    TD3_TRY_RC(td3_radix_sort_u32(k0, k1, v0, v1, e, bits_for(n_nodes), &ko, &vo, w.base + w.used,
                                  w.size - w.used, s));
    // the row offsets from the boundaries between equal keys of the sorted entries; valid
    // entries sort before the invalid key n_nodes (row_start[n_nodes] of them), the entries
    // after them are widened too (partners holds e slots), so no host read
    TD3_TRY(td3_launch_chained(k_csr_out, td3_blocks(e + 1, 256), 256, 0, s, vo, ko, e, n_nodes,
                               row_start, partners, entry_row));
    TD3_CHECK_LAUNCH();
    return TD3_OK;
}
