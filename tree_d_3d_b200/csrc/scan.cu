// Device-wide exclusive scans and a stable LSD radix sort, the integer building
// blocks of the tree build, the traversal and the interaction-list CSR rows.
#include "common.cuh"

namespace {

constexpr int SCAN_THREADS = 256;
constexpr int SCAN_ITEMS = 8;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

template <typename T>
__device__ __forceinline__ T shfl_up(T v, int d) {
    return __shfl_up_sync(0xffffffffu, v, d);
}
template <>
__device__ __forceinline__ td3_i64x2 shfl_up<td3_i64x2>(td3_i64x2 v, int d) {
    td3_i64x2 o;
    o.a = __shfl_up_sync(0xffffffffu, v.a, d);
    o.b = __shfl_up_sync(0xffffffffu, v.b, d);
    return o;
}

template <typename T>
__device__ __forceinline__ T warp_inclusive(T v) {
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        T o = shfl_up(v, d);
        if ((threadIdx.x & 31) >= d) v += o;
    }
    return v;
}

// Exclusive block scan of one value per thread; returns the exclusive prefix and the
// block total in *total.
template <typename T>
__device__ __forceinline__ T block_exclusive(T v, T* total) {
    __shared__ T warp_sums[32];
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    T inc = warp_inclusive(v);
    if (lane == 31) warp_sums[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        int nw = (blockDim.x + 31) >> 5;
        T s = lane < nw ? warp_sums[lane] : T(0);
        s = warp_inclusive(s);
        if (lane < nw) warp_sums[lane] = s;
    }
    __syncthreads();
    T warp_off = warp ? warp_sums[warp - 1] : T(0);
    *total = warp_sums[((blockDim.x + 31) >> 5) - 1];
    __syncthreads();
    return warp_off + inc - v;
}

template <typename T>
__global__ void k_tile_reduce(const T* __restrict__ in, i64 n, T* __restrict__ partial) {
    td3_chain_wait();
    td3_chain_release();
    i64 base = (i64)blockIdx.x * SCAN_TILE;
    T s = 0;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i) {
        i64 k = base + (i64)i * SCAN_THREADS + threadIdx.x;
        if (k < n) s += in[k];
    }
    T total;
    block_exclusive(s, &total);
    if (threadIdx.x == 0) partial[blockIdx.x] = total;
}

// One block scans the partials in place (exclusive), carrying across chunks.
template <typename T>
__global__ void k_partials_scan(T* partial, i64 m, T* total_out) {
    td3_chain_wait();
    td3_chain_release();
    T carry = 0;
    for (i64 base = 0; base < m; base += blockDim.x) {
        i64 k = base + threadIdx.x;
        T v = k < m ? partial[k] : T(0);
        T tot;
        T ex = block_exclusive(v, &tot);
        if (k < m) partial[k] = carry + ex;
        carry += tot;
    }
    if (threadIdx.x == 0 && total_out) *total_out = carry;
}

template <typename T>
__global__ void k_tile_scan(const T* __restrict__ in, T* __restrict__ out, i64 n,
                            const T* __restrict__ partial) {
    td3_chain_wait();
    td3_chain_release();
    i64 base = (i64)blockIdx.x * SCAN_TILE + (i64)threadIdx.x * SCAN_ITEMS;
    T v[SCAN_ITEMS];
    T s = 0;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i) {
        i64 k = base + i;
        v[i] = k < n ? in[k] : T(0);
        s += v[i];
    }
    T total;
    T off = block_exclusive(s, &total) + partial[blockIdx.x];
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i) {
        i64 k = base + i;
        if (k < n) out[k] = off;
        off += v[i];
    }
}

// Arrays of one tile: the whole scan in one block, one launch.
template <typename T>
__global__ void k_single_tile_scan(const T* __restrict__ in, T* __restrict__ out, i64 n,
                                   T* __restrict__ total_out) {
    td3_chain_wait();
    td3_chain_release();
    i64 base = (i64)threadIdx.x * SCAN_ITEMS;
    T v[SCAN_ITEMS];
    T s = 0;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i) {
        i64 k = base + i;
        v[i] = k < n ? in[k] : T(0);
        s += v[i];
    }
    T total;
    T off = block_exclusive(s, &total);
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i) {
        i64 k = base + i;
        if (k < n) out[k] = off;
        off += v[i];
    }
    if (threadIdx.x == 0 && total_out) *total_out = total;
}

template <typename T>
int exclusive_scan(const T* in, T* out, i64 n, T* total, void* ws, size_t ws_bytes,
                   cudaStream_t stream) {
    if (n <= 0) {
        if (total) TD3_TRY(cudaMemsetAsync(total, 0, sizeof(T), stream));
        return TD3_OK;
    }
    if (n <= SCAN_TILE) {
        TD3_TRY(td3_launch_chained(k_single_tile_scan<T>, 1, SCAN_THREADS, 0, stream, in, out, n,
                                   total));
        return TD3_OK;
    }
    i64 tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    if ((size_t)tiles * sizeof(T) > ws_bytes) return TD3_EWORKSPACE;
    T* partial = static_cast<T*>(ws);
    TD3_TRY(td3_launch_chained(k_tile_reduce<T>, (unsigned)tiles, SCAN_THREADS, 0, stream, in, n,
                               partial));
    TD3_TRY(td3_launch_chained(k_partials_scan<T>, 1, 1024, 0, stream, partial, tiles, total));
    TD3_TRY(td3_launch_chained(k_tile_scan<T>, (unsigned)tiles, SCAN_THREADS, 0, stream, in, out,
                               n, (const T*)partial));
    return TD3_OK;
}

// ------------------------------------------------------------------- radix sort
// Stable LSD radix sort of uint32 keys with uint32 values, 8-bit digits.  A pass is a
// per-tile digit histogram, an exclusive scan of the (digit-major) histograms, and a
// scatter.  A tile is 8 warps x 512 consecutive items; a warp ranks its items round by
// round (32 consecutive items per round) with __match_any_sync, so equal digits keep
// input order; the tile is then reordered by digit in shared memory and written out in
// runs of equal digits (coalesced stores).
constexpr int SORT_THREADS = 256;
constexpr int SORT_WARPS = SORT_THREADS / 32;
constexpr int SORT_ITEMS = 8;
constexpr int WARP_ITEMS = 32 * SORT_ITEMS;
constexpr int SORT_TILE = SORT_THREADS * SORT_ITEMS;
constexpr int RADIX_BITS = 8;
constexpr int RADIX = 1 << RADIX_BITS;
static_assert(RADIX == SORT_THREADS, "one thread per digit in the tile totals");

__device__ __forceinline__ unsigned lanes_below() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

__global__ void __launch_bounds__(SORT_THREADS)
k_sort_hist(const unsigned* __restrict__ keys, i64 n, int shift, unsigned mask, int n_tiles,
            int* __restrict__ hist) {
    __shared__ int counts[SORT_WARPS][RADIX];
    td3_chain_wait();
    td3_chain_release();
    for (int i = threadIdx.x; i < SORT_WARPS * RADIX; i += SORT_THREADS) (&counts[0][0])[i] = 0;
    __syncthreads();
    int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    i64 base = (i64)blockIdx.x * SORT_TILE + (i64)wib * WARP_ITEMS;
    // the warp's items loaded first, then counted with shared-memory atomics into the
    // warp's own counts (lanes that meet on a digit are serialised by the hardware)
    unsigned dig[SORT_ITEMS];
#pragma unroll
    for (int r = 0; r < SORT_ITEMS; ++r) {
        i64 k = base + r * 32 + lane;
        dig[r] = k < n ? (keys[k] >> shift) & mask : RADIX;
    }
#pragma unroll
    for (int r = 0; r < SORT_ITEMS; ++r)
        if (dig[r] < RADIX) atomicAdd(&counts[wib][dig[r]], 1);
    __syncthreads();
    int d = threadIdx.x, sum = 0;
#pragma unroll
    for (int w = 0; w < SORT_WARPS; ++w) sum += counts[w][d];
    hist[(i64)d * n_tiles + blockIdx.x] = sum;
}

__global__ void __launch_bounds__(SORT_THREADS)
k_sort_scatter(const unsigned* __restrict__ keys, const unsigned* __restrict__ vals,
               unsigned* __restrict__ keys_out, unsigned* __restrict__ vals_out, i64 n, int shift,
               unsigned mask, int n_tiles, const int* __restrict__ offsets) {
    __shared__ unsigned skeys[SORT_TILE];
    __shared__ unsigned svals[SORT_TILE];
    __shared__ int wcount[SORT_WARPS][RADIX];
    __shared__ int tstart[RADIX];
    __shared__ int goff[RADIX];
    td3_chain_wait();
    td3_chain_release();
    for (int i = threadIdx.x; i < SORT_WARPS * RADIX; i += SORT_THREADS) (&wcount[0][0])[i] = 0;
    __syncthreads();
    int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    i64 tile = (i64)blockIdx.x * SORT_TILE;
    i64 base = tile + (i64)wib * WARP_ITEMS;
    unsigned kr[SORT_ITEMS], vr[SORT_ITEMS];
    int rank[SORT_ITEMS];
    unsigned below = lanes_below();
#pragma unroll
    for (int r = 0; r < SORT_ITEMS; ++r) {
        i64 k = base + r * 32 + lane;
        bool live = k < n;
        kr[r] = live ? keys[k] : 0u;
        vr[r] = live ? vals[k] : 0u;
        unsigned d = live ? (kr[r] >> shift) & mask : RADIX;
        unsigned peers = __match_any_sync(0xffffffffu, d);
        int before = __popc(peers & below);
        int seen = live ? wcount[wib][d] : 0;
        __syncwarp();
        if (live && before == 0) wcount[wib][d] = seen + __popc(peers);
        __syncwarp();
        rank[r] = seen + before;
    }
    __syncthreads();
    // digit d (thread d): per-warp exclusive offsets within the digit, the tile total
    int d = threadIdx.x, sum = 0;
#pragma unroll
    for (int w = 0; w < SORT_WARPS; ++w) {
        int c = wcount[w][d];
        wcount[w][d] = sum;
        sum += c;
    }
    int total;
    int start = block_exclusive(sum, &total);
    tstart[d] = start;
    goff[d] = offsets[(i64)d * n_tiles + blockIdx.x];
    __syncthreads();
#pragma unroll
    for (int r = 0; r < SORT_ITEMS; ++r) {
        if (base + r * 32 + lane < n) {
            int dg = (int)((kr[r] >> shift) & mask);
            int at = tstart[dg] + wcount[wib][dg] + rank[r];
            skeys[at] = kr[r];
            svals[at] = vr[r];
        }
    }
    __syncthreads();
    int count = (int)(n - tile < SORT_TILE ? n - tile : SORT_TILE);
    for (int i = threadIdx.x; i < count; i += SORT_THREADS) {
        unsigned key = skeys[i];
        int dg = (int)((key >> shift) & mask);
        i64 p = (i64)goff[dg] + (i - tstart[dg]);
        keys_out[p] = key;
        vals_out[p] = svals[i];
    }
}

int radix_sort(unsigned* keys, unsigned* keys_alt, unsigned* vals, unsigned* vals_alt, i64 n,
               int bits, unsigned** keys_out, unsigned** vals_out, void* ws, size_t ws_bytes,
               cudaStream_t stream) {
    *keys_out = keys;
    *vals_out = vals;
    if (n <= 1 || bits <= 0) return TD3_OK;
    if (n > 0x7fffffffLL) return TD3_EINVAL;
    int n_tiles = (int)((n + SORT_TILE - 1) / SORT_TILE);
    i64 n_hist = (i64)RADIX * n_tiles;
    if (n_hist > 0x7fffffffLL) return TD3_EINVAL;
    Workspace w(ws, ws_bytes);
    int* hist = w.take<int>(n_hist);
    void* scan_ws = w.base + w.used;
    size_t scan_bytes = w.size - w.used;
    if (!hist) return TD3_EWORKSPACE;
    unsigned *src_k = keys, *dst_k = keys_alt, *src_v = vals, *dst_v = vals_alt;
    if (bits > 32) bits = 32;
    for (int shift = 0; shift < bits; shift += RADIX_BITS) {
        int digit_bits = bits - shift < RADIX_BITS ? bits - shift : RADIX_BITS;
        unsigned mask = (1u << digit_bits) - 1u;
        TD3_TRY(td3_launch_chained(k_sort_hist, n_tiles, SORT_THREADS, 0, stream,
                                   (const unsigned*)src_k, n, shift, mask, n_tiles, hist));
        TD3_TRY_RC(td3_exclusive_scan_i32(hist, hist, n_hist, nullptr, scan_ws, scan_bytes, stream));
        TD3_TRY(td3_launch_chained(k_sort_scatter, n_tiles, SORT_THREADS, 0, stream,
                                   (const unsigned*)src_k, (const unsigned*)src_v, dst_k, dst_v,
                                   n, shift, mask, n_tiles, (const int*)hist));
        TD3_CHECK_LAUNCH();
        unsigned* tk = src_k;
        src_k = dst_k;
        dst_k = tk;
        unsigned* tv = src_v;
        src_v = dst_v;
        dst_v = tv;
    }
    *keys_out = src_k;
    *vals_out = src_v;
    return TD3_OK;
}

}  // namespace

size_t td3_scan_workspace(i64 n) {
    i64 tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    return td3_ws_bytes<td3_i64x2>(tiles + 1);
}

int td3_exclusive_scan_i64(const i64* in, i64* out, i64 n, i64* total, void* ws, size_t ws_bytes,
                           cudaStream_t stream) {
    return exclusive_scan<i64>(in, out, n, total, ws, ws_bytes, stream);
}

int td3_exclusive_scan_i32(const int* in, int* out, i64 n, int* total, void* ws, size_t ws_bytes,
                           cudaStream_t stream) {
    return exclusive_scan<int>(in, out, n, total, ws, ws_bytes, stream);
}

int td3_exclusive_scan_i64x2(const td3_i64x2* in, td3_i64x2* out, i64 n, td3_i64x2* total,
                             void* ws, size_t ws_bytes, cudaStream_t stream) {
    return exclusive_scan<td3_i64x2>(in, out, n, total, ws, ws_bytes, stream);
}

size_t td3_sort_workspace(i64 n) {
    i64 n_tiles = (n + SORT_TILE - 1) / SORT_TILE;
    i64 n_hist = (i64)RADIX * n_tiles;
    return td3_ws_bytes<int>(n_hist) + td3_scan_workspace(n_hist);
}

int td3_radix_sort_u32(unsigned* keys, unsigned* keys_alt, unsigned* vals, unsigned* vals_alt,
                       i64 n, int bits, unsigned** keys_out, unsigned** vals_out, void* ws,
                       size_t ws_bytes, cudaStream_t stream) {
    return radix_sort(keys, keys_alt, vals, vals_alt, n, bits, keys_out, vals_out, ws, ws_bytes,
                      stream);
}

// ------------------------------------------------------------------- C ABI
extern "C" size_t td3_radix_sort_workspace_size(int64_t n) { return td3_sort_workspace(n); }

extern "C" int td3_radix_sort_pairs(uint32_t* keys, uint32_t* keys_alt, uint32_t* values,
                                    uint32_t* values_alt, int64_t n, int bits, int* result_in_alt,
                                    void* workspace, size_t workspace_bytes, void* stream) {
    unsigned *ko, *vo;
    int rc = td3_radix_sort_u32(keys, keys_alt, values, values_alt, n, bits, &ko, &vo, workspace,
                                workspace_bytes, td3_stream(stream));
    if (result_in_alt) *result_in_alt = (ko != keys);
    return rc;
}
