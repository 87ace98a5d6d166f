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
        k_single_tile_scan<T><<<1, SCAN_THREADS, 0, stream>>>(in, out, n, total);
        TD3_CHECK_LAUNCH();
        return TD3_OK;
    }
    i64 tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    if ((size_t)tiles * sizeof(T) > ws_bytes) return TD3_EWORKSPACE;
    T* partial = static_cast<T*>(ws);
    k_tile_reduce<T><<<(unsigned)tiles, SCAN_THREADS, 0, stream>>>(in, n, partial);
    k_partials_scan<T><<<1, 1024, 0, stream>>>(partial, tiles, total);
    k_tile_scan<T><<<(unsigned)tiles, SCAN_THREADS, 0, stream>>>(in, out, n, partial);
    TD3_CHECK_LAUNCH();
    return TD3_OK;
}

// ------------------------------------------------------------------- radix sort
constexpr int SORT_THREADS = 256;
constexpr int SORT_ITEMS = 8;
constexpr int SORT_TILE = SORT_THREADS * SORT_ITEMS;
constexpr int RADIX_BITS = 4;
constexpr int RADIX = 1 << RADIX_BITS;

template <typename K>
__global__ void k_sort_hist(const K* __restrict__ keys, i64 n, int shift, int n_tiles,
                            int* __restrict__ hist) {
    __shared__ int counts[RADIX];
    if (threadIdx.x < RADIX) counts[threadIdx.x] = 0;
    __syncthreads();
    i64 base = (i64)blockIdx.x * SORT_TILE;
    for (int i = threadIdx.x; i < SORT_TILE; i += SORT_THREADS) {
        i64 k = base + i;
        if (k < n) atomicAdd(&counts[(int)((keys[k] >> shift) & (RADIX - 1))], 1);
    }
    __syncthreads();
    if (threadIdx.x < RADIX) hist[threadIdx.x * n_tiles + blockIdx.x] = counts[threadIdx.x];
}

// Each thread owns SORT_ITEMS consecutive items of the tile; an item's rank in the
// tile is (items of smaller digits) + (same digit in earlier threads) + (same digit
// earlier in this thread), which keeps equal keys in input order (stable).
template <typename K>
__global__ void k_sort_scatter(const K* __restrict__ keys, const unsigned* __restrict__ vals,
                               K* __restrict__ keys_out, unsigned* __restrict__ vals_out,
                               i64 n, int shift, int n_tiles, const int* __restrict__ offsets) {
    __shared__ int table[RADIX * SORT_THREADS];
    __shared__ K skeys[SORT_TILE];
    __shared__ unsigned svals[SORT_TILE];
    i64 base = (i64)blockIdx.x * SORT_TILE;
    for (int i = threadIdx.x; i < SORT_TILE; i += SORT_THREADS) {
        i64 k = base + i;
        if (k < n) {
            skeys[i] = keys[k];
            svals[i] = vals[k];
        }
    }
    __syncthreads();
    int local[RADIX];
#pragma unroll
    for (int d = 0; d < RADIX; ++d) local[d] = 0;
    int first = threadIdx.x * SORT_ITEMS;
#pragma unroll
    for (int i = 0; i < SORT_ITEMS; ++i) {
        if (base + first + i < n) {
            int d = (int)((skeys[first + i] >> shift) & (RADIX - 1));
#pragma unroll
            for (int e = 0; e < RADIX; ++e) local[e] += (e == d);
        }
    }
#pragma unroll
    for (int d = 0; d < RADIX; ++d) table[d * SORT_THREADS + threadIdx.x] = local[d];
    __syncthreads();
    // exclusive scan of table (digit-major): thread t owns entries [16 t, 16 t + 16)
    int run[RADIX];
    int s = 0;
#pragma unroll
    for (int i = 0; i < RADIX; ++i) {
        run[i] = table[threadIdx.x * RADIX + i];
        s += run[i];
    }
    int total;
    int off = block_exclusive(s, &total);
#pragma unroll
    for (int i = 0; i < RADIX; ++i) {
        table[threadIdx.x * RADIX + i] = off;
        off += run[i];
    }
    __syncthreads();
    int pos[RADIX];
#pragma unroll
    for (int d = 0; d < RADIX; ++d)
        pos[d] = table[d * SORT_THREADS + threadIdx.x] - table[d * SORT_THREADS] +
                 offsets[d * n_tiles + blockIdx.x];
#pragma unroll
    for (int i = 0; i < SORT_ITEMS; ++i) {
        if (base + first + i < n) {
            K key = skeys[first + i];
            int d = (int)((key >> shift) & (RADIX - 1));
            int p = 0;
#pragma unroll
            for (int e = 0; e < RADIX; ++e)
                if (e == d) p = pos[e]++;
            keys_out[p] = key;
            vals_out[p] = svals[first + i];
        }
    }
}

template <typename K>
int radix_sort(K* keys, K* keys_alt, unsigned* vals, unsigned* vals_alt, i64 n, int bits,
               K** keys_out, unsigned** vals_out, void* ws, size_t ws_bytes,
               cudaStream_t stream) {
    *keys_out = keys;
    *vals_out = vals;
    if (n <= 1 || bits <= 0) return TD3_OK;
    if (n > 0x7fffffffLL) return TD3_EINVAL;
    int n_tiles = (int)((n + SORT_TILE - 1) / SORT_TILE);
    i64 n_hist = (i64)RADIX * n_tiles;
    Workspace w(ws, ws_bytes);
    int* hist = w.take<int>(n_hist);
    void* scan_ws = w.base + w.used;
    size_t scan_bytes = w.size - w.used;
    if (!hist) return TD3_EWORKSPACE;
    K* src_k = keys;
    K* dst_k = keys_alt;
    unsigned* src_v = vals;
    unsigned* dst_v = vals_alt;
    for (int shift = 0; shift < bits; shift += RADIX_BITS) {
        k_sort_hist<K><<<n_tiles, SORT_THREADS, 0, stream>>>(src_k, n, shift, n_tiles, hist);
        TD3_TRY_RC(td3_exclusive_scan_i32(hist, hist, n_hist, nullptr, scan_ws, scan_bytes, stream));
        k_sort_scatter<K><<<n_tiles, SORT_THREADS, 0, stream>>>(src_k, src_v, dst_k, dst_v, n,
                                                                shift, n_tiles, hist);
        TD3_CHECK_LAUNCH();
        K* tk = src_k;
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
    return radix_sort<unsigned>(keys, keys_alt, vals, vals_alt, n, bits, keys_out, vals_out, ws,
                                ws_bytes, stream);
}

int td3_radix_sort_u64(unsigned long long* keys, unsigned long long* keys_alt, unsigned* vals,
                       unsigned* vals_alt, i64 n, int bits, unsigned long long** keys_out,
                       unsigned** vals_out, void* ws, size_t ws_bytes, cudaStream_t stream) {
    return radix_sort<unsigned long long>(keys, keys_alt, vals, vals_alt, n, bits, keys_out,
                                          vals_out, ws, ws_bytes, stream);
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
