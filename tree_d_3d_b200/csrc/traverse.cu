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
// predicates use exactly rounded operations (this file is compiled with --fmad=false).
#include "common.cuh"

namespace {

constexpr int TRAV_THREADS = 256;

struct Pair {
    i64 a, b;
};

enum : int { ACT_NONE = 0, ACT_M2L = 1, ACT_P2P = 2, ACT_SELF = 3, ACT_SPLIT_A = 4, ACT_SPLIT_B = 5 };

// The decision of the mutual traversal for pair (a, b) (fmm_traverse_pyccel.py:48-106).
__device__ __forceinline__ int classify_mutual(i64 a, i64 b, const double* __restrict__ center,
                                               const double* __restrict__ half,
                                               const i64* __restrict__ start,
                                               const i64* __restrict__ end,
                                               const i64* __restrict__ child, double theta) {
    if (end[a] == start[a] || end[b] == start[b]) return ACT_NONE;
    bool leaf_a = child[a] < 0, leaf_b = child[b] < 0;
    if (a == b) return leaf_a ? ACT_P2P : ACT_SELF;
    double dx = xsub(center[2 * a], center[2 * b]);
    double dy = xsub(center[2 * a + 1], center[2 * b + 1]);
    double distance = xsqrt(xnorm2(dx, dy));
    double radii = xmul(TD3_ROOT2, xadd(half[a], half[b]));
    if (radii < xmul(theta, distance)) return ACT_M2L;
    if (leaf_a && leaf_b) return ACT_P2P;
    if (leaf_b || (!leaf_a && half[a] >= half[b])) return ACT_SPLIT_A;
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

__global__ void k_trav_classify(const Pair* __restrict__ frontier, i64 nf,
                                const double* __restrict__ center, const double* __restrict__ half,
                                const i64* __restrict__ start, const i64* __restrict__ end,
                                const i64* __restrict__ child, double theta,
                                signed char* __restrict__ action, td3_i64x2* __restrict__ counts) {
    i64 k = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nf) return;
    Pair pr = frontier[k];
    int act = classify_mutual(pr.a, pr.b, center, half, start, end, child, theta);
    action[k] = (signed char)act;
    counts[k] = action_counts(act);
}

__global__ void k_trav_emit(const Pair* __restrict__ frontier, i64 nf,
                            const signed char* __restrict__ action,
                            const td3_i64x2* __restrict__ offsets, const i64* __restrict__ child,
                            i64 base_m2l, i64 base_p2p, Pair* __restrict__ m2l,
                            Pair* __restrict__ p2p, Pair* __restrict__ next) {
    i64 k = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nf) return;
    int act = action[k];
    if (act == ACT_NONE) return;
    Pair pr = frontier[k];
    td3_i64x2 off = offsets[k];
    switch (act) {
        case ACT_M2L: m2l[base_m2l + (off.a & 0xffffffffLL)] = pr; break;
        case ACT_P2P: p2p[base_p2p + (off.a >> 32)] = pr; break;
        case ACT_SELF: {
            i64 first = child[pr.a], i = off.b;
            for (int c = 0; c < 4; ++c)
                for (int d = c; d < 4; ++d) next[i++] = Pair{first + c, first + d};
            break;
        }
        case ACT_SPLIT_A: {
            i64 first = child[pr.a];
            for (int c = 0; c < 4; ++c) next[off.b + c] = Pair{first + c, pr.b};
            break;
        }
        case ACT_SPLIT_B: {
            i64 first = child[pr.b];
            for (int c = 0; c < 4; ++c) next[off.b + c] = Pair{pr.a, first + c};
            break;
        }
    }
}

__global__ void k_root_pair(Pair* frontier) { frontier[0] = Pair{0, 0}; }

// ------------------------------------------------------------------ dual traversal
// One-way decision for (target cell a, source cell b) (dual_traverse_pyccel.py:46-86).
__global__ void k_dual_classify(const Pair* __restrict__ frontier, i64 nf,
                                const double* __restrict__ t_center, const double* __restrict__ t_half,
                                const i64* __restrict__ t_start, const i64* __restrict__ t_end,
                                const i64* __restrict__ t_child,
                                const double* __restrict__ s_center, const double* __restrict__ s_half,
                                const i64* __restrict__ s_start, const i64* __restrict__ s_end,
                                const i64* __restrict__ s_child, double theta,
                                signed char* __restrict__ action, td3_i64x2* __restrict__ counts) {
    i64 k = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nf) return;
    Pair pr = frontier[k];
    i64 a = pr.a, b = pr.b;
    int act;
    if (t_end[a] == t_start[a] || s_end[b] == s_start[b]) {
        act = ACT_NONE;
    } else {
        double dx = xsub(t_center[2 * a], s_center[2 * b]);
        double dy = xsub(t_center[2 * a + 1], s_center[2 * b + 1]);
        if (xmul(TD3_ROOT2, xadd(t_half[a], s_half[b])) < xmul(theta, xsqrt(xnorm2(dx, dy)))) {
            act = ACT_M2L;
        } else {
            bool leaf_a = t_child[a] < 0, leaf_b = s_child[b] < 0;
            if (leaf_a && leaf_b)
                act = ACT_P2P;
            else if (leaf_b || (!leaf_a && t_half[a] >= s_half[b]))
                act = ACT_SPLIT_A;
            else
                act = ACT_SPLIT_B;
        }
    }
    action[k] = (signed char)act;
    counts[k] = action_counts(act);
}

__global__ void k_dual_emit(const Pair* __restrict__ frontier, i64 nf,
                            const signed char* __restrict__ action,
                            const td3_i64x2* __restrict__ offsets, const i64* __restrict__ t_child,
                            const i64* __restrict__ s_child, i64 base_m2l, i64 base_p2p,
                            Pair* __restrict__ m2l, Pair* __restrict__ p2p, Pair* __restrict__ next) {
    i64 k = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nf) return;
    int act = action[k];
    if (act == ACT_NONE) return;
    Pair pr = frontier[k];
    td3_i64x2 off = offsets[k];
    if (act == ACT_M2L) {
        m2l[base_m2l + (off.a & 0xffffffffLL)] = pr;
    } else if (act == ACT_P2P) {
        p2p[base_p2p + (off.a >> 32)] = pr;
    } else if (act == ACT_SPLIT_A) {
        i64 first = t_child[pr.a];
        for (int c = 0; c < 4; ++c) next[off.b + c] = Pair{first + c, pr.b};
    } else {
        i64 first = s_child[pr.b];
        for (int c = 0; c < 4; ++c) next[off.b + c] = Pair{pr.a, first + c};
    }
}

struct TraverseBuffers {
    Pair* frontier[2];
    signed char* action;
    td3_i64x2* counts;
    td3_i64x2* total;
    void* scan_ws;
    size_t scan_bytes;
};

size_t traverse_workspace(i64 frontier_cap) {
    return 2 * td3_ws_bytes<Pair>(frontier_cap) + td3_ws_bytes<signed char>(frontier_cap) +
           td3_ws_bytes<td3_i64x2>(frontier_cap) + td3_ws_bytes<td3_i64x2>(1) +
           td3_scan_workspace(frontier_cap) + 256;
}

bool take_traverse(Workspace& w, i64 frontier_cap, TraverseBuffers& b) {
    b.frontier[0] = w.take<Pair>(frontier_cap);
    b.frontier[1] = w.take<Pair>(frontier_cap);
    b.action = w.take<signed char>(frontier_cap);
    b.counts = w.take<td3_i64x2>(frontier_cap);
    b.total = w.take<td3_i64x2>(1);
    if (!b.total) return false;
    b.scan_ws = w.base + w.used;
    b.scan_bytes = w.size - w.used;
    return true;
}

// ------------------------------------------------------------------ pair CSR
__global__ void k_csr_keys(const Pair* __restrict__ pairs, i64 count, int mutual, unsigned invalid,
                           unsigned* __restrict__ keys, unsigned* __restrict__ vals,
                           i64* __restrict__ row_count) {
    i64 p = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= count) return;
    Pair pr = pairs[p];
    if (mutual) {
        keys[2 * p] = (unsigned)pr.a;
        vals[2 * p] = (unsigned)pr.b;
        atomicAdd(reinterpret_cast<unsigned long long*>(row_count + pr.a), 1ULL);
        if (pr.a != pr.b) {
            keys[2 * p + 1] = (unsigned)pr.b;
            vals[2 * p + 1] = (unsigned)pr.a;
            atomicAdd(reinterpret_cast<unsigned long long*>(row_count + pr.b), 1ULL);
        } else {
            keys[2 * p + 1] = invalid;
            vals[2 * p + 1] = 0;
        }
    } else {
        keys[p] = (unsigned)pr.a;
        vals[p] = (unsigned)pr.b;
        atomicAdd(reinterpret_cast<unsigned long long*>(row_count + pr.a), 1ULL);
    }
}

__global__ void k_widen_vals(const unsigned* __restrict__ in, i64 count, i64* __restrict__ out) {
    i64 k = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < count) out[k] = in[k];
}

int bits_for(i64 v) {
    int b = 1;
    while (b < 32 && ((i64)1 << b) <= v) ++b;
    return b;
}

}  // namespace

extern "C" size_t td3_fmm_traverse_workspace_size(int64_t frontier_capacity) {
    return traverse_workspace(frontier_capacity);
}

extern "C" int td3_fmm_traverse(const double* node_center, const double* node_half,
                                const int64_t* node_start, const int64_t* node_end,
                                const int64_t* node_child, double theta, int64_t* m2l,
                                int64_t m2l_capacity, int64_t* p2p, int64_t p2p_capacity,
                                int64_t frontier_capacity, int64_t* sizes, void* workspace,
                                size_t workspace_bytes, void* stream) {
    if (frontier_capacity < 1 || m2l_capacity < 0 || p2p_capacity < 0) return TD3_EINVAL;
    cudaStream_t s = td3_stream(stream);
    Workspace w(workspace, workspace_bytes);
    TraverseBuffers b;
    if (!take_traverse(w, frontier_capacity, b)) return TD3_EWORKSPACE;
    Pair* pm2l = reinterpret_cast<Pair*>(m2l);
    Pair* pp2p = reinterpret_cast<Pair*>(p2p);
    k_root_pair<<<1, 1, 0, s>>>(b.frontier[0]);
    TD3_CHECK_LAUNCH();
    i64 nf = 1, n_m2l = 0, n_p2p = 0;
    int cur = 0;
    sizes[0] = sizes[1] = sizes[2] = sizes[3] = 0;
    while (nf > 0) {
        unsigned nb = td3_blocks(nf, TRAV_THREADS);
        k_trav_classify<<<nb, TRAV_THREADS, 0, s>>>(b.frontier[cur], nf, node_center, node_half,
                                                    node_start, node_end, node_child, theta,
                                                    b.action, b.counts);
        TD3_TRY_RC(td3_exclusive_scan_i64x2(b.counts, b.counts, nf, b.total, b.scan_ws,
                                            b.scan_bytes, s));
        td3_i64x2 tot;
        TD3_TRY(cudaMemcpyAsync(&tot, b.total, sizeof(tot), cudaMemcpyDeviceToHost, s));
        TD3_TRY(cudaStreamSynchronize(s));
        i64 add_m2l = tot.a & 0xffffffffLL, add_p2p = tot.a >> 32, nn = tot.b;
        if (n_m2l + add_m2l > m2l_capacity || n_p2p + add_p2p > p2p_capacity ||
            nn > frontier_capacity) {
            sizes[0] = n_m2l + add_m2l;
            sizes[1] = n_p2p + add_p2p;
            sizes[2] = nn;
            sizes[3] = -1;
            return TD3_ENEEDMORE;
        }
        k_trav_emit<<<nb, TRAV_THREADS, 0, s>>>(b.frontier[cur], nf, b.action, b.counts,
                                                node_child, n_m2l, n_p2p, pm2l, pp2p,
                                                b.frontier[cur ^ 1]);
        TD3_CHECK_LAUNCH();
        n_m2l += add_m2l;
        n_p2p += add_p2p;
        nf = nn;
        cur ^= 1;
    }
    sizes[0] = n_m2l;
    sizes[1] = n_p2p;
    return TD3_OK;
}

extern "C" int td3_dual_traverse(const double* t_center, const double* t_half,
                                 const int64_t* t_start, const int64_t* t_end,
                                 const int64_t* t_child, const double* s_center,
                                 const double* s_half, const int64_t* s_start,
                                 const int64_t* s_end, const int64_t* s_child, double theta,
                                 int64_t* m2l, int64_t m2l_capacity, int64_t* p2p,
                                 int64_t p2p_capacity, int64_t frontier_capacity, int64_t* sizes,
                                 void* workspace, size_t workspace_bytes, void* stream) {
    if (frontier_capacity < 1 || m2l_capacity < 0 || p2p_capacity < 0) return TD3_EINVAL;
    cudaStream_t s = td3_stream(stream);
    Workspace w(workspace, workspace_bytes);
    TraverseBuffers b;
    if (!take_traverse(w, frontier_capacity, b)) return TD3_EWORKSPACE;
    Pair* pm2l = reinterpret_cast<Pair*>(m2l);
    Pair* pp2p = reinterpret_cast<Pair*>(p2p);
    k_root_pair<<<1, 1, 0, s>>>(b.frontier[0]);
    TD3_CHECK_LAUNCH();
    i64 nf = 1, n_m2l = 0, n_p2p = 0;
    int cur = 0;
    sizes[0] = sizes[1] = sizes[2] = sizes[3] = 0;
    while (nf > 0) {
        unsigned nb = td3_blocks(nf, TRAV_THREADS);
        k_dual_classify<<<nb, TRAV_THREADS, 0, s>>>(b.frontier[cur], nf, t_center, t_half, t_start,
                                                    t_end, t_child, s_center, s_half, s_start,
                                                    s_end, s_child, theta, b.action, b.counts);
        TD3_TRY_RC(td3_exclusive_scan_i64x2(b.counts, b.counts, nf, b.total, b.scan_ws,
                                            b.scan_bytes, s));
        td3_i64x2 tot;
        TD3_TRY(cudaMemcpyAsync(&tot, b.total, sizeof(tot), cudaMemcpyDeviceToHost, s));
        TD3_TRY(cudaStreamSynchronize(s));
        i64 add_m2l = tot.a & 0xffffffffLL, add_p2p = tot.a >> 32, nn = tot.b;
        if (n_m2l + add_m2l > m2l_capacity || n_p2p + add_p2p > p2p_capacity ||
            nn > frontier_capacity) {
            sizes[0] = n_m2l + add_m2l;
            sizes[1] = n_p2p + add_p2p;
            sizes[2] = nn;
            sizes[3] = -1;
            return TD3_ENEEDMORE;
        }
        k_dual_emit<<<nb, TRAV_THREADS, 0, s>>>(b.frontier[cur], nf, b.action, b.counts, t_child,
                                                s_child, n_m2l, n_p2p, pm2l, pp2p,
                                                b.frontier[cur ^ 1]);
        TD3_CHECK_LAUNCH();
        n_m2l += add_m2l;
        n_p2p += add_p2p;
        nf = nn;
        cur ^= 1;
    }
    sizes[0] = n_m2l;
    sizes[1] = n_p2p;
    return TD3_OK;
}

extern "C" size_t td3_pair_csr_workspace_size(int64_t count, int mutual, int64_t n_nodes) {
    i64 e = mutual ? 2 * count : count;
    size_t sort = td3_sort_workspace(e), scan = td3_scan_workspace(n_nodes + 1);
    return 4 * td3_ws_bytes<unsigned>(e) + (sort > scan ? sort : scan);
}

extern "C" int td3_pair_csr(const int64_t* pairs, int64_t count, int mutual, int64_t n_nodes,
                            int64_t* row_start, int64_t* partners, void* workspace,
                            size_t workspace_bytes, void* stream) {
    if (count < 0 || n_nodes < 1 || n_nodes >= 0x7fffffffLL) return TD3_EINVAL;
    cudaStream_t s = td3_stream(stream);
    TD3_TRY(cudaMemsetAsync(row_start, 0, sizeof(i64) * (n_nodes + 1), s));
    if (count == 0) return TD3_OK;
    i64 e = mutual ? 2 * count : count;
    Workspace w(workspace, workspace_bytes);
    unsigned* k0 = w.take<unsigned>(e);
    unsigned* k1 = w.take<unsigned>(e);
    unsigned* v0 = w.take<unsigned>(e);
    unsigned* v1 = w.take<unsigned>(e);
    if (!v1) return TD3_EWORKSPACE;
    // row counts go to row_start[1..], then an exclusive scan in place makes offsets
    k_csr_keys<<<td3_blocks(count, 256), 256, 0, s>>>(reinterpret_cast<const Pair*>(pairs), count,
                                                      mutual, (unsigned)n_nodes, k0, v0, row_start);
    TD3_CHECK_LAUNCH();
    unsigned *ko, *vo;
    TD3_TRY_RC(td3_radix_sort_u32(k0, k1, v0, v1, e, bits_for(n_nodes), &ko, &vo, w.base + w.used,
                                  w.size - w.used, s));
    TD3_TRY_RC(td3_exclusive_scan_i64(row_start, row_start, n_nodes + 1, nullptr, w.base + w.used,
                                      w.size - w.used, s));
    // valid entries sort before the invalid key n_nodes (row_start[n_nodes] of them); the
    // entries after them are widened too (partners holds e slots), so no host read
    k_widen_vals<<<td3_blocks(e, 256), 256, 0, s>>>(vo, e, partners);
    TD3_CHECK_LAUNCH();
    return TD3_OK;
}
