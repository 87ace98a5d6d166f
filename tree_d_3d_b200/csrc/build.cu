// The quadtree build: bit-identical to the reference's breadth-first build
// (K/quadtree_build/quadtree_build_pyccel.py:12-137 and its GPU level path
// ft:532-625), as a GPU MSD radix sort with one 2-bit Morton digit per level.
//
// Level d holds the nodes levels[d]..levels[d+1].  Per level:
//   1. split flags of the level's nodes (count > leaf_capacity, depth < max_depth),
//      exclusive scan -> each splitting node's rank, children numbered hi + 4 * rank
//      (breadth first, in the order of their parents);
//   2. the children's geometry: half = 0.5 * parent half, centres parent -/+ half
//      (the same floating-point operations as the reference, hence the same values);
//   3. the quadrant digit of every particle slot in a splitting node, from the
//      comparisons x > cx and y < cy against its node's centre;
//   4. an exclusive scan of the slots' one-hot digits (four counts in two words):
//      the children's ranges, and each slot's rank among its node's slots of the
//      same digit;
//   5. a stable scatter of the slots (permutation, positions, node of each slot).
// A stable partition per level keeps each leaf's particles in input order, as the
// reference.  This file is compiled with --fmad=false.
#include "common.cuh"

namespace {

constexpr int BUILD_THREADS = 256;

__global__ void k_build_init(const double* __restrict__ pos, i64 n, double* __restrict__ spos,
                             i64* __restrict__ perm, int* __restrict__ slot_node,
                             double xmid, double ymid, double half, double* node_center,
                             double* node_half, i64* node_start, i64* node_end, i64* node_depth) {
    i64 k = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) {
        spos[k] = pos[k];
        spos[n + k] = pos[n + k];
        perm[k] = k;
        slot_node[k] = 0;
    }
    if (k == 0) {
        node_center[0] = xmid;
        node_center[1] = ymid;
        node_half[0] = half;
        node_start[0] = 0;
        node_end[0] = n;
        node_depth[0] = 0;
    }
}

__global__ void k_split_flags(i64 lo, i64 hi, i64 leaf_capacity, i64 max_depth,
                              const i64* __restrict__ node_start, const i64* __restrict__ node_end,
                              const i64* __restrict__ node_depth, i64* __restrict__ flags) {
    i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    i64 node = lo + t;
    if (node >= hi) return;
    flags[t] = (node_end[node] - node_start[node] > leaf_capacity && node_depth[node] < max_depth)
                   ? 1 : 0;
}

__global__ void k_children(i64 lo, i64 hi, const i64* __restrict__ flags,
                           const i64* __restrict__ rank, double* __restrict__ node_center,
                           double* __restrict__ node_half, i64* __restrict__ node_child,
                           i64* __restrict__ node_depth) {
    i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    i64 node = lo + t;
    if (node >= hi) return;
    if (!flags[t]) {
        node_child[node] = -1;
        return;
    }
    i64 first = hi + 4 * rank[t];
    node_child[node] = first;
    double half = 0.5 * node_half[node];
    double cx = node_center[2 * node], cy = node_center[2 * node + 1];
    i64 depth = node_depth[node] + 1;
    for (int c = 0; c < 4; ++c) {
        node_half[first + c] = half;
        node_depth[first + c] = depth;
    }
    // children 0..3: upper left, upper right, lower left, lower right
    node_center[2 * first] = cx - half;
    node_center[2 * first + 1] = cy + half;
    node_center[2 * (first + 1)] = cx + half;
    node_center[2 * (first + 1) + 1] = cy + half;
    node_center[2 * (first + 2)] = cx - half;
    node_center[2 * (first + 2) + 1] = cy - half;
    node_center[2 * (first + 3)] = cx + half;
    node_center[2 * (first + 3) + 1] = cy - half;
}

// One-hot quadrant digit of each slot, packed (q0 + q1 << 32, q2 + q3 << 32); zero
// for slots of nodes that do not split.  digit[k] is -1 for those.
__global__ void k_digits(i64 n, const double* __restrict__ spos, const int* __restrict__ slot_node,
                         const double* __restrict__ node_center, const i64* __restrict__ node_child,
                         signed char* __restrict__ digit, td3_i64x2* __restrict__ onehot) {
    i64 k = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    int node = slot_node[k];
    td3_i64x2 v(0, 0);
    int q = -1;
    if (node_child[node] >= 0) {
        q = (spos[k] > node_center[2 * node] ? 1 : 0) + (spos[n + k] < node_center[2 * node + 1] ? 2 : 0);
        i64 one = (q & 1) ? ((i64)1 << 32) : (i64)1;
        if (q < 2)
            v.a = one;
        else
            v.b = one;
    }
    digit[k] = (signed char)q;
    onehot[k] = v;
}

__device__ __forceinline__ i64 field_of(const td3_i64x2& v, int q) {
    i64 w = (q < 2) ? v.a : v.b;
    return (q & 1) ? (w >> 32) : (w & 0xffffffffLL);
}

__device__ __forceinline__ td3_i64x2 prefix_at(const td3_i64x2* __restrict__ pre, i64 k, i64 n,
                                               const td3_i64x2* __restrict__ total) {
    return k < n ? pre[k] : *total;
}

__global__ void k_child_ranges(i64 lo, i64 hi, i64 n, const i64* __restrict__ flags,
                               const i64* __restrict__ node_child, i64* __restrict__ node_start,
                               i64* __restrict__ node_end, const td3_i64x2* __restrict__ pre,
                               const td3_i64x2* __restrict__ total) {
    i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    i64 node = lo + t;
    if (node >= hi || !flags[t]) return;
    i64 s = node_start[node], e = node_end[node];
    td3_i64x2 cnt = prefix_at(pre, e, n, total) - prefix_at(pre, s, n, total);
    i64 first = node_child[node];
    i64 start = s;
    for (int q = 0; q < 4; ++q) {
        i64 size = field_of(cnt, q);
        node_start[first + q] = start;
        node_end[first + q] = start + size;
        start += size;
    }
}

__global__ void k_scatter(i64 n, const signed char* __restrict__ digit,
                          const td3_i64x2* __restrict__ pre, const int* __restrict__ slot_node,
                          const i64* __restrict__ node_child, const i64* __restrict__ node_start,
                          const i64* __restrict__ perm, const double* __restrict__ spos,
                          i64* __restrict__ new_perm, double* __restrict__ new_spos,
                          int* __restrict__ new_slot_node) {
    i64 k = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    int q = digit[k];
    int node = slot_node[k];
    i64 slot = k;
    int new_node = node;
    if (q >= 0) {
        i64 child = node_child[node] + q;
        i64 s = node_start[node];
        // rank among the node's slots of digit q that come before k
        i64 rank = field_of(pre[k], q) - field_of(pre[s], q);
        slot = node_start[child] + rank;
        new_node = (int)child;
    }
    new_perm[slot] = perm[k];
    new_spos[slot] = spos[k];
    new_spos[n + slot] = spos[n + k];
    new_slot_node[slot] = new_node;
}

struct BuildBuffers {
    int* slot[2];
    i64* perm_tmp;
    double* spos_tmp;
    signed char* digit;
    td3_i64x2* onehot;
    td3_i64x2* onehot_total;
    i64* flags;
    i64* rank;
    i64* n_split;
    void* scan_ws;
    size_t scan_bytes;
};

size_t build_workspace(i64 n, i64 capacity) {
    i64 m = n > capacity ? n : capacity;
    return 2 * td3_ws_bytes<int>(n) + td3_ws_bytes<i64>(n) + td3_ws_bytes<double>(2 * n) +
           td3_ws_bytes<signed char>(n) + td3_ws_bytes<td3_i64x2>(n) + td3_ws_bytes<td3_i64x2>(1) +
           2 * td3_ws_bytes<i64>(capacity) + td3_ws_bytes<i64>(1) + td3_scan_workspace(m) + 256;
}

}  // namespace

extern "C" size_t td3_quadtree_build_workspace_size(int64_t n, int64_t capacity) {
    return build_workspace(n, capacity);
}

extern "C" int td3_quadtree_build(const double* pos, int64_t n, double xmid, double ymid,
                                  double half, int64_t leaf_capacity, int64_t max_depth,
                                  int64_t capacity, double* node_center, double* node_half,
                                  int64_t* node_start, int64_t* node_end, int64_t* node_child,
                                  int64_t* node_depth, int64_t* perm, double* sorted_pos,
                                  int64_t* levels, int64_t* sizes, void* workspace,
                                  size_t workspace_bytes, void* stream) {
    if (n < 1 || n > 0x7fffffffLL || leaf_capacity < 1 || max_depth < 0 || capacity < 1)
        return TD3_EINVAL;
    cudaStream_t s = td3_stream(stream);
    Workspace w(workspace, workspace_bytes);
    BuildBuffers b;
    b.slot[0] = w.take<int>(n);
    b.slot[1] = w.take<int>(n);
    b.perm_tmp = w.take<i64>(n);
    b.spos_tmp = w.take<double>(2 * n);
    b.digit = w.take<signed char>(n);
    b.onehot = w.take<td3_i64x2>(n);
    b.onehot_total = w.take<td3_i64x2>(1);
    b.flags = w.take<i64>(capacity);
    b.rank = w.take<i64>(capacity);
    b.n_split = w.take<i64>(1);
    if (!b.n_split) return TD3_EWORKSPACE;
    b.scan_ws = w.base + w.used;
    b.scan_bytes = w.size - w.used;

    i64* perm_cur = perm;
    i64* perm_alt = b.perm_tmp;
    double* spos_cur = sorted_pos;
    double* spos_alt = b.spos_tmp;
    int* slot_cur = b.slot[0];
    int* slot_alt = b.slot[1];
    k_build_init<<<td3_blocks(n, BUILD_THREADS), BUILD_THREADS, 0, s>>>(
        pos, n, spos_cur, perm_cur, slot_cur, xmid, ymid, half, node_center, node_half, node_start,
        node_end, node_depth);
    TD3_CHECK_LAUNCH();
    levels[0] = 0;
    levels[1] = 1;
    i64 n_levels = 1, lo = 0, hi = 1;
    sizes[2] = 0;
    for (;;) {
        i64 count_level = hi - lo;
        unsigned nb = td3_blocks(count_level, BUILD_THREADS);
        k_split_flags<<<nb, BUILD_THREADS, 0, s>>>(lo, hi, leaf_capacity, max_depth, node_start,
                                                   node_end, node_depth, b.flags);
        TD3_TRY_RC(td3_exclusive_scan_i64(b.flags, b.rank, count_level, b.n_split, b.scan_ws,
                                          b.scan_bytes, s));
        i64 n_split = 0;
        TD3_TRY(cudaMemcpyAsync(&n_split, b.n_split, sizeof(i64), cudaMemcpyDeviceToHost, s));
        TD3_TRY(cudaStreamSynchronize(s));
        i64 count = hi + 4 * n_split;
        if (count > capacity) {
            sizes[0] = hi;
            sizes[1] = n_levels;
            sizes[2] = 1;
            return TD3_ENEEDMORE;
        }
        k_children<<<nb, BUILD_THREADS, 0, s>>>(lo, hi, b.flags, b.rank, node_center, node_half,
                                                node_child, node_depth);
        TD3_CHECK_LAUNCH();
        if (n_split == 0) break;
        unsigned pb = td3_blocks(n, BUILD_THREADS);
        k_digits<<<pb, BUILD_THREADS, 0, s>>>(n, spos_cur, slot_cur, node_center, node_child,
                                              b.digit, b.onehot);
        TD3_TRY_RC(td3_exclusive_scan_i64x2(b.onehot, b.onehot, n, b.onehot_total, b.scan_ws,
                                            b.scan_bytes, s));
        k_child_ranges<<<nb, BUILD_THREADS, 0, s>>>(lo, hi, n, b.flags, node_child, node_start,
                                                    node_end, b.onehot, b.onehot_total);
        k_scatter<<<pb, BUILD_THREADS, 0, s>>>(n, b.digit, b.onehot, slot_cur, node_child,
                                               node_start, perm_cur, spos_cur, perm_alt, spos_alt,
                                               slot_alt);
        TD3_CHECK_LAUNCH();
        i64* tp = perm_cur;
        perm_cur = perm_alt;
        perm_alt = tp;
        double* ts = spos_cur;
        spos_cur = spos_alt;
        spos_alt = ts;
        int* tn = slot_cur;
        slot_cur = slot_alt;
        slot_alt = tn;
        lo = hi;
        hi = count;
        n_levels += 1;
        levels[n_levels] = hi;
    }
    if (perm_cur != perm) {
        TD3_TRY(cudaMemcpyAsync(perm, perm_cur, sizeof(i64) * n, cudaMemcpyDeviceToDevice, s));
        TD3_TRY(cudaMemcpyAsync(sorted_pos, spos_cur, sizeof(double) * 2 * n,
                                cudaMemcpyDeviceToDevice, s));
    }
    sizes[0] = hi;
    sizes[1] = n_levels;
    return TD3_OK;
}
