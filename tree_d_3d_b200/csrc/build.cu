// The quadtree build: bit-identical to the reference's breadth-first build
// (K/quadtree_build/quadtree_build_pyccel.py:12-137 and its GPU level path
// ft:532-625).  Two forms give the same arrays:
//   - from sorted quadrant paths (build_by_keys, below): one host read for the whole
//     tree; used whenever 32 digits of path suffice;
//   - level by level, a GPU MSD radix sort with one 2-bit digit per level, for deeper
//     trees (clusters finer than 2^-32 of the root).
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

size_t level_workspace(i64 n, i64 capacity) {
    i64 m = n > capacity ? n : capacity;
    return 2 * td3_ws_bytes<int>(n) + td3_ws_bytes<i64>(n) + td3_ws_bytes<double>(2 * n) +
           td3_ws_bytes<signed char>(n) + td3_ws_bytes<td3_i64x2>(n) + td3_ws_bytes<td3_i64x2>(1) +
           2 * td3_ws_bytes<i64>(capacity) + td3_ws_bytes<i64>(1) + td3_scan_workspace(m) + 256;
}

// ---------------------------------------------------------------------------------
// The same tree from sorted quadrant paths.  Every particle's path (its quadrant digit
// at each depth, from the centre chain the build itself computes) is a key of up to 32
// digits, first digit highest.  Sorted stably, the particles of any node are a
// contiguous run, so for the run starting at sorted position j at depth d:
//   j starts a run at depth d    <=>  j == 0 or cpl(key[j-1], key[j]) < d,
//   the run holds > C particles  <=>  cpl(key[j], key[j+C]) >= d,
// (cpl: common leading digits), and the splitting nodes that start at j are the depths
// a_j < d <= b_j, a_j = cpl(key[j-1], key[j]), b_j = min(cpl(key[j], key[j+C]),
// max_depth - 1).  Their count per depth gives the level sizes (one read by the host);
// each splitting node then writes its own first-child index and its four children,
// numbered as the breadth-first build numbers them (level offset + 4 x the parent's
// rank among the level's splitting nodes + quadrant).  A last stable sort by leaf
// restores input order inside each leaf.  The first sort uses the leading 16 digits
// only; a tree that splits deeper is sorted again on 32 digits, and one deeper still
// is built level by level.
constexpr int KEY_DIGITS = 32;
constexpr int PREFIX_DIGITS = 16;

struct KeyLevels {
    i64 levels[KEY_DIGITS + 2];  // first node of each level
    i64 dstart[KEY_DIGITS + 1];  // first splitting node of each depth in the depth-sorted list
};

struct KeySummary {
    int invalid;      // 1: a position is not finite, 2: a position lies outside the root
    int deeper;       // a node at the last key digit still splits
    i64 split_total;  // splitting nodes
    int count[KEY_DIGITS];
};

constexpr int INVALID_NONFINITE = 1;
constexpr int INVALID_OUTSIDE = 2;

__device__ __forceinline__ int key_cpl(unsigned long long a, unsigned long long b, int digits) {
    unsigned long long x = a ^ b;
    if (x == 0) return digits;
    int top = 63 - __clzll((long long)x);
    return digits - 1 - (top >> 1);
}

// digit i (1-based, first digit = 1) of a key of `digits` digits
__device__ __forceinline__ int key_digit(unsigned long long key, int i, int digits) {
    return (int)((key >> (2 * (digits - i))) & 3ULL);
}

__global__ void k_path_keys(const double* __restrict__ pos, i64 n, double xmid, double ymid,
                            double half, int digits, int prefix_shift,
                            unsigned long long* __restrict__ key, unsigned* __restrict__ prefix,
                            unsigned* __restrict__ index, KeySummary* summary) {
    i64 k = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    double x = pos[k], y = pos[n + k];
    // the inputs the reference rejects (ft:788-794): not finite, or outside the root
    if (!(isfinite(x) && isfinite(y)))
        atomicOr(&summary->invalid, INVALID_NONFINITE);
    else if (x < xmid - half || x > xmid + half || y < ymid - half || y > ymid + half)
        atomicOr(&summary->invalid, INVALID_OUTSIDE);
    double cx = xmid, cy = ymid, h = half;
    unsigned long long v = 0;
    for (int d = 0; d < digits; ++d) {
        int q = (x > cx ? 1 : 0) + (y < cy ? 2 : 0);
        v = (v << 2) | (unsigned long long)q;
        h = 0.5 * h;
        cx = (q & 1) ? cx + h : cx - h;
        cy = (q & 2) ? cy - h : cy + h;
    }
    key[k] = v;
    prefix[k] = (unsigned)(v >> prefix_shift);
    index[k] = (unsigned)k;
}

__global__ void k_gather_keys(i64 n, const unsigned long long* __restrict__ key,
                              const unsigned* __restrict__ index, int shift,
                              unsigned long long* __restrict__ out) {
    i64 j = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (j < n) out[j] = key[index[j]] >> shift;
}

__global__ void k_low_digits(i64 n, const unsigned long long* __restrict__ key, int bits,
                             unsigned* __restrict__ low, unsigned* __restrict__ index) {
    i64 k = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    low[k] = (unsigned)(key[k] & ((1ULL << bits) - 1ULL));
    index[k] = (unsigned)k;
}

__global__ void k_gather_high(i64 n, const unsigned long long* __restrict__ key,
                              const unsigned* __restrict__ index, int shift,
                              unsigned* __restrict__ high) {
    i64 j = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (j < n) high[j] = (unsigned)(key[index[j]] >> shift);
}

__global__ void k_split_depths(const unsigned long long* __restrict__ skey, i64 n, int digits,
                               i64 capacity_c, i64 max_depth, signed char* __restrict__ first,
                               i64* __restrict__ len, KeySummary* summary) {
    __shared__ int cnt[KEY_DIGITS];
    if (threadIdx.x < KEY_DIGITS) cnt[threadIdx.x] = 0;
    __syncthreads();
    i64 j = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (j < n) {
        int a = j == 0 ? -1 : key_cpl(skey[j - 1], skey[j], digits);
        int b = -1;
        if (capacity_c < n - j) {
            b = key_cpl(skey[j], skey[j + capacity_c], digits);
            if ((i64)b > max_depth - 1) b = (int)(max_depth - 1);
        }
        if (b >= digits) {
            atomicOr(&summary->deeper, 1);
            b = digits - 1;
        }
        first[j] = (signed char)a;
        len[j] = b > a ? b - a : 0;
        for (int d = a + 1; d <= b; ++d) atomicAdd(&cnt[d], 1);
    }
    __syncthreads();
    if (threadIdx.x < KEY_DIGITS && cnt[threadIdx.x]) atomicAdd(&summary->count[threadIdx.x], cnt[threadIdx.x]);
}

__global__ void k_expand_splits(i64 n, const signed char* __restrict__ first,
                                const i64* __restrict__ len, const i64* __restrict__ offset,
                                unsigned* __restrict__ depth, unsigned* __restrict__ start) {
    i64 j = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    i64 o = offset[j];
    int a = first[j];
    for (i64 t = 0; t < len[j]; ++t) {
        depth[o + t] = (unsigned)(a + 1 + t);
        start[o + t] = (unsigned)j;
    }
}

__global__ void k_key_root(double xmid, double ymid, double half, i64 n, int root_splits,
                           double* node_center, double* node_half, i64* node_start,
                           i64* node_end, i64* node_child, i64* node_depth, int* leaf_flag) {
    node_center[0] = xmid;
    node_center[1] = ymid;
    node_half[0] = half;
    node_start[0] = 0;
    node_end[0] = n;
    node_depth[0] = 0;
    if (!root_splits) {
        node_child[0] = -1;
        leaf_flag[0] = 1;
    }
}

__global__ void k_key_nodes(i64 n_split, const unsigned* __restrict__ sdepth,
                            const unsigned* __restrict__ sstart,
                            const unsigned long long* __restrict__ skey, i64 n, int digits,
                            const KeyLevels L, double xmid, double ymid, double half,
                            i64 capacity_c, i64 max_depth, double* __restrict__ node_center,
                            double* __restrict__ node_half, i64* __restrict__ node_start,
                            i64* __restrict__ node_end, i64* __restrict__ node_child,
                            i64* __restrict__ node_depth, int* __restrict__ leaf_flag) {
    i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_split) return;
    int d = (int)sdepth[t];
    i64 j = sstart[t];
    i64 rank = t - L.dstart[d];
    unsigned long long key = skey[j];
    i64 id = 0;
    if (d > 0) {
        // the parent: the last splitting node of depth d - 1 starting at or before j
        i64 lo = L.dstart[d - 1], hi = L.dstart[d] - 1;
        while (lo < hi) {
            i64 mid = (lo + hi + 1) >> 1;
            if ((i64)sstart[mid] <= j) lo = mid;
            else hi = mid - 1;
        }
        id = L.levels[d] + 4 * (lo - L.dstart[d - 1]) + key_digit(key, d, digits);
    }
    i64 first = L.levels[d + 1] + 4 * rank;
    node_child[id] = first;
    // the node's geometry by the build's own chain of centres
    double cx = xmid, cy = ymid, h = half;
    for (int i = 1; i <= d; ++i) {
        int q = key_digit(key, i, digits);
        h = 0.5 * h;
        cx = (q & 1) ? cx + h : cx - h;
        cy = (q & 2) ? cy - h : cy + h;
    }
    // the end of the node's run: the first position past j with fewer than d common digits
    i64 lo = j + 1, hi = n;
    while (lo < hi) {
        i64 mid = (lo + hi) >> 1;
        if (key_cpl(key, skey[mid], digits) >= d) lo = mid + 1;
        else hi = mid;
    }
    i64 s[5];
    s[0] = j;
    s[4] = lo;
    for (int q = 1; q < 4; ++q) {
        i64 a = s[q - 1], b = s[4];
        while (a < b) {
            i64 mid = (a + b) >> 1;
            if (key_digit(skey[mid], d + 1, digits) < q) a = mid + 1;
            else b = mid;
        }
        s[q] = a;
    }
    double hc = 0.5 * h;
    for (int q = 0; q < 4; ++q) {
        i64 c = first + q;
        node_center[2 * c] = (q & 1) ? cx + hc : cx - hc;
        node_center[2 * c + 1] = (q & 2) ? cy - hc : cy + hc;
        node_half[c] = hc;
        node_depth[c] = d + 1;
        node_start[c] = s[q];
        node_end[c] = s[q + 1];
        i64 count = s[q + 1] - s[q];
        if (!(count > capacity_c && d + 1 < max_depth)) {
            node_child[c] = -1;
            if (count > 0) leaf_flag[s[q]] = 1;
        }
    }
}

// leaf ordinal of each particle, scattered to input order
__global__ void k_leaf_keys(i64 n, const int* __restrict__ flag, const int* __restrict__ excl,
                            const unsigned* __restrict__ index, unsigned* __restrict__ leaf,
                            unsigned* __restrict__ iota) {
    i64 j = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    leaf[index[j]] = (unsigned)(excl[j] + flag[j] - 1);
    iota[j] = (unsigned)j;
}

__global__ void k_key_finish(i64 n, const unsigned* __restrict__ order,
                             const double* __restrict__ pos, i64* __restrict__ perm,
                             double* __restrict__ sorted_pos) {
    i64 j = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    i64 k = order[j];
    perm[j] = k;
    sorted_pos[j] = pos[k];
    sorted_pos[n + j] = pos[n + k];
}

int bits_of(i64 v) {
    int b = 1;
    while (b < 32 && ((i64)1 << b) <= v) ++b;
    return b;
}

struct KeyBuffers {
    unsigned long long* key;
    unsigned long long* skey;
    unsigned *u0, *u1, *v0, *v1;
    signed char* first;
    i64* len;
    i64* offset;
    int* flag;
    int* excl;
    unsigned *sd0, *sd1, *ss0, *ss1;
    KeySummary* summary;
    void* tail;
    size_t tail_bytes;
};

size_t key_workspace(i64 n, i64 capacity) {
    i64 splits = capacity / 4 + 1;
    i64 m = n > splits ? n : splits;
    size_t sort = td3_sort_workspace(m), scan = td3_scan_workspace(n);
    return 2 * td3_ws_bytes<unsigned long long>(n) + 4 * td3_ws_bytes<unsigned>(n) +
           td3_ws_bytes<signed char>(n) + 2 * td3_ws_bytes<i64>(n) + 2 * td3_ws_bytes<int>(n) +
           4 * td3_ws_bytes<unsigned>(splits) + td3_ws_bytes<KeySummary>(1) +
           (sort > scan ? sort : scan) + 256;
}

bool take_keys(Workspace& w, i64 n, i64 capacity, KeyBuffers& b) {
    i64 splits = capacity / 4 + 1;
    b.key = w.take<unsigned long long>(n);
    b.skey = w.take<unsigned long long>(n);
    b.u0 = w.take<unsigned>(n);
    b.u1 = w.take<unsigned>(n);
    b.v0 = w.take<unsigned>(n);
    b.v1 = w.take<unsigned>(n);
    b.first = w.take<signed char>(n);
    b.len = w.take<i64>(n);
    b.offset = w.take<i64>(n);
    b.flag = w.take<int>(n);
    b.excl = w.take<int>(n);
    b.sd0 = w.take<unsigned>(splits);
    b.sd1 = w.take<unsigned>(splits);
    b.ss0 = w.take<unsigned>(splits);
    b.ss1 = w.take<unsigned>(splits);
    b.summary = w.take<KeySummary>(1);
    if (!b.summary) return false;
    b.tail = w.base + w.used;
    b.tail_bytes = w.size - w.used;
    return true;
}

// Sorted keys of `digits` digits and the split summary (one host read).  keys: the
// particles' paths of `total` digits.
int key_pass(const KeyBuffers& b, i64 n, int total, int digits, i64 leaf_capacity,
             i64 max_depth, KeySummary& host, cudaStream_t s) {
    unsigned nb = td3_blocks(n, BUILD_THREADS);
    unsigned *ko, *vo;
    if (digits <= PREFIX_DIGITS) {
        // b.u0 holds the leading `digits` digits, b.v0 the particle indices
        TD3_TRY_RC(td3_radix_sort_u32(b.u0, b.u1, b.v0, b.v1, n, 2 * digits, &ko, &vo, b.tail,
                                      b.tail_bytes, s));
    } else {
        int low_bits = 2 * (digits - PREFIX_DIGITS);
        k_low_digits<<<nb, BUILD_THREADS, 0, s>>>(n, b.key, low_bits, b.u0, b.v0);
        TD3_TRY_RC(td3_radix_sort_u32(b.u0, b.u1, b.v0, b.v1, n, low_bits, &ko, &vo, b.tail,
                                      b.tail_bytes, s));
        unsigned* high = ko == b.u0 ? b.u1 : b.u0;
        unsigned* high_alt = ko == b.u0 ? b.u0 : b.u1;
        unsigned* idx_alt = vo == b.v0 ? b.v1 : b.v0;
        k_gather_high<<<nb, BUILD_THREADS, 0, s>>>(n, b.key, vo, low_bits, high);
        TD3_TRY_RC(td3_radix_sort_u32(high, high_alt, vo, idx_alt, n, 2 * PREFIX_DIGITS, &ko, &vo,
                                      b.tail, b.tail_bytes, s));
    }
    k_gather_keys<<<nb, BUILD_THREADS, 0, s>>>(n, b.key, vo, 2 * (total - digits), b.skey);
    if (vo != b.v0)
        TD3_TRY(cudaMemcpyAsync(b.v0, vo, sizeof(unsigned) * n, cudaMemcpyDeviceToDevice, s));
    // clear all but `invalid`, which the path-key pass wrote
    TD3_TRY(cudaMemsetAsync(&b.summary->deeper, 0, sizeof(KeySummary) - offsetof(KeySummary, deeper),
                            s));
    k_split_depths<<<nb, BUILD_THREADS, 0, s>>>(b.skey, n, digits, leaf_capacity, max_depth,
                                                b.first, b.len, b.summary);
    TD3_CHECK_LAUNCH();
    TD3_TRY_RC(td3_exclusive_scan_i64(b.len, b.offset, n, &b.summary->split_total, b.tail,
                                      b.tail_bytes, s));
    TD3_TRY(cudaMemcpyAsync(&host, b.summary, sizeof(KeySummary), cudaMemcpyDeviceToHost, s));
    TD3_TRY(cudaStreamSynchronize(s));
    return TD3_OK;
}

// TD3_OK with *levelwise = true when the tree needs more than KEY_DIGITS digits.
int build_by_keys(const double* pos, i64 n, double xmid, double ymid, double half,
                  i64 leaf_capacity, i64 max_depth, i64 capacity, double* node_center,
                  double* node_half, i64* node_start, i64* node_end, i64* node_child,
                  i64* node_depth, i64* perm, double* sorted_pos, i64* levels, i64* sizes,
                  Workspace& w, cudaStream_t s, bool* levelwise) {
    *levelwise = false;
    KeyBuffers b;
    if (!take_keys(w, n, capacity, b)) return TD3_EWORKSPACE;
    int total = max_depth < KEY_DIGITS ? (int)max_depth : KEY_DIGITS;
    int digits = total < PREFIX_DIGITS ? total : PREFIX_DIGITS;
    unsigned nb = td3_blocks(n, BUILD_THREADS);
    TD3_TRY(cudaMemsetAsync(&b.summary->invalid, 0, sizeof(int), s));
    k_path_keys<<<nb, BUILD_THREADS, 0, s>>>(pos, n, xmid, ymid, half, total, 2 * (total - digits),
                                             b.key, b.u0, b.v0, b.summary);
    TD3_CHECK_LAUNCH();
    KeySummary host;
    TD3_TRY_RC(key_pass(b, n, total, digits, leaf_capacity, max_depth, host, s));
    if (host.invalid) {
        sizes[3] = (host.invalid & INVALID_NONFINITE) ? 1 : 2;
        return TD3_EINVAL;
    }
    if (host.deeper && digits < total) {
        digits = total;
        TD3_TRY_RC(key_pass(b, n, total, digits, leaf_capacity, max_depth, host, s));
    }
    if (host.deeper) {
        *levelwise = true;
        return TD3_OK;
    }
    // level offsets: level 0 is the root, level d + 1 the children of depth d's splits
    KeyLevels L;
    int depth = 0;  // deepest level
    for (int d = 0; d < KEY_DIGITS; ++d)
        if (host.count[d] > 0) depth = d + 1;
    L.levels[0] = 0;
    L.levels[1] = 1;
    L.dstart[0] = 0;
    for (int d = 0; d < KEY_DIGITS; ++d) {
        L.dstart[d + 1] = L.dstart[d] + host.count[d];
        L.levels[d + 2] = L.levels[d + 1] + 4 * (i64)host.count[d];
    }
    i64 node_count = L.levels[depth + 1];
    if (node_count > capacity) {
        sizes[0] = node_count;
        sizes[1] = depth + 1;
        sizes[2] = 1;
        return TD3_ENEEDMORE;
    }
    i64 n_split = host.split_total;
    TD3_TRY(cudaMemsetAsync(b.flag, 0, sizeof(int) * n, s));
    k_key_root<<<1, 1, 0, s>>>(xmid, ymid, half, n, n_split > 0, node_center, node_half,
                               node_start, node_end, node_child, node_depth, b.flag);
    if (n_split > 0) {
        unsigned sb = td3_blocks(n_split, BUILD_THREADS);
        k_expand_splits<<<nb, BUILD_THREADS, 0, s>>>(n, b.first, b.len, b.offset, b.sd0, b.ss0);
        unsigned *dso, *sso;
        TD3_TRY_RC(td3_radix_sort_u32(b.sd0, b.sd1, b.ss0, b.ss1, n_split, bits_of(depth), &dso,
                                      &sso, b.tail, b.tail_bytes, s));
        k_key_nodes<<<sb, BUILD_THREADS, 0, s>>>(n_split, dso, sso, b.skey, n, digits, L, xmid,
                                                 ymid, half, leaf_capacity, max_depth, node_center,
                                                 node_half, node_start, node_end, node_child,
                                                 node_depth, b.flag);
        TD3_CHECK_LAUNCH();
    }
    // input order inside each leaf: a stable sort of the input indices by leaf ordinal
    TD3_TRY_RC(td3_exclusive_scan_i32(b.flag, b.excl, n, nullptr, b.tail, b.tail_bytes, s));
    k_leaf_keys<<<nb, BUILD_THREADS, 0, s>>>(n, b.flag, b.excl, b.v0, b.u0, b.v1);
    TD3_CHECK_LAUNCH();
    unsigned *lo_k, *lo_v;
    TD3_TRY_RC(td3_radix_sort_u32(b.u0, b.u1, b.v1, b.v0, n, bits_of(n), &lo_k, &lo_v, b.tail,
                                  b.tail_bytes, s));
    k_key_finish<<<nb, BUILD_THREADS, 0, s>>>(n, lo_v, pos, perm, sorted_pos);
    TD3_CHECK_LAUNCH();
    for (int d = 0; d <= depth + 1; ++d) levels[d] = L.levels[d];
    sizes[0] = node_count;
    sizes[1] = depth + 1;
    sizes[2] = 0;
    return TD3_OK;
}

size_t build_workspace(i64 n, i64 capacity) {
    size_t a = level_workspace(n, capacity), b = key_workspace(n, capacity);
    return a > b ? a : b;
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
    sizes[3] = 0;
    {
        Workspace wk(workspace, workspace_bytes);
        bool levelwise = false;
        int rc = build_by_keys(pos, n, xmid, ymid, half, leaf_capacity, max_depth, capacity,
                               node_center, node_half, node_start, node_end, node_child,
                               node_depth, perm, sorted_pos, levels, sizes, wk, s, &levelwise);
        if (rc != TD3_OK || !levelwise) return rc;
    }
    // deeper than the keys hold: level by level
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
