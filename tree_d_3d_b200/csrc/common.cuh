// Shared definitions of the sm_100a kernels of the tree-d-3d field solver.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "treed3d.h"

typedef int64_t i64;

#define TD3_CHECK_LAUNCH()                                   \
    do {                                                     \
        cudaError_t e_ = cudaGetLastError();                 \
        if (e_ != cudaSuccess) return td3_cuda_error(e_);    \
    } while (0)

#define TD3_TRY(expr)                                        \
    do {                                                     \
        cudaError_t e_ = (expr);                             \
        if (e_ != cudaSuccess) return td3_cuda_error(e_);    \
    } while (0)

#define TD3_TRY_RC(expr)                                     \
    do {                                                     \
        int rc_ = (expr);                                    \
        if (rc_ != TD3_OK) return rc_;                       \
    } while (0)

// Records the CUDA error for td3_last_error and maps it to TD3_ECUDA.
int td3_cuda_error(cudaError_t err);

// Records a message for td3_last_error.
void td3_set_error(const char* message);

static inline cudaStream_t td3_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

static inline unsigned td3_blocks(i64 n, int threads) {
    i64 b = (n + threads - 1) / threads;
    return (unsigned)(b < 1 ? 1 : b);
}

// Programmatic dependent launch for chains of short dependent kernels (a level or a
// traversal generation at a time): the launch may start while the previous kernel on
// the stream still runs; the kernel's first statement is td3_chain_wait(), which
// returns once every earlier kernel of the stream has finished and its memory writes
// are visible (hardware-tracked, griddepcontrol.wait), and td3_chain_release() lets the
// next kernel of the chain start launching.
__device__ __forceinline__ void td3_chain_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void td3_chain_release() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

template <typename... Params, typename... Args>
static inline cudaError_t td3_launch_chained(void (*kernel)(Params...), unsigned grid,
                                             unsigned block, size_t smem, cudaStream_t s,
                                             Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, static_cast<Params>(args)...);
}

// Carves aligned sub-buffers out of a caller-provided workspace.
struct Workspace {
    char* base;
    size_t size;
    size_t used;
    __host__ Workspace(void* p, size_t n) : base(static_cast<char*>(p)), size(n), used(0) {}
    template <typename T>
    __host__ T* take(i64 count) {
        size_t bytes = ((size_t)(count > 0 ? count : 1) * sizeof(T) + 255) & ~(size_t)255;
        if (used + bytes > size) return nullptr;
        T* out = reinterpret_cast<T*>(base + used);
        used += bytes;
        return out;
    }
};

// Bytes of a workspace sub-buffer of `count` items of T (as Workspace::take rounds it).
template <typename T>
static inline size_t td3_ws_bytes(i64 count) {
    return ((size_t)(count > 0 ? count : 1) * sizeof(T) + 255) & ~(size_t)255;
}

// ---------------------------------------------------------------------------------
// Exactly rounded arithmetic for the decisions the reference takes (opening tests,
// traversal predicates).  nvcc would contract a*b+c into one FMA; these intrinsics
// are never contracted, so each operation rounds as in the reference's CPU code.
__device__ __forceinline__ double xmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double xadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double xsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double xsqrt(double a) { return __dsqrt_rn(a); }

// |r|^2 = rx*rx + ry*ry, each product rounded, then the sum rounded.
__device__ __forceinline__ double xnorm2(double rx, double ry) {
    return xadd(xmul(rx, rx), xmul(ry, ry));
}

// Compensated (Kahan) FP32 sum of the mixed-precision kernels: the running error c is
// subtracted from each new term; value() returns the sum in FP64.
struct KahanF {
    float s = 0.0f, c = 0.0f;
    __device__ __forceinline__ void add(float x) {
        float y = x - c;
        float t = s + y;
        c = (t - s) - y;
        s = t;
    }
    __device__ __forceinline__ double value() const { return (double)s - (double)c; }
};

// Pairs per node row of the size-scaled FP32 moments (td3_scale_moments): order + 1
// rounded up to even, so every row starts on a 16-byte boundary.
__host__ __device__ __forceinline__ int td3_hat_width(int order) { return (order + 2) & ~1; }

// Pairs 2c and 2c + 1 of a scaled-moment row, zero beyond the order (w = order + 1).
__device__ __forceinline__ float4 td3_hat_pair(const float2* row, int c, int w) {
    return 2 * c < w ? reinterpret_cast<const float4*>(row)[c] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
}

// ln(x) for x > 0 of any FP64 magnitude in FP32 arithmetic: x = f 2^e with f in [0.5, 1)
// (frexp, exact), ln x = ln f + e ln 2.
__device__ __forceinline__ float log_split(double x) {
    int e;
    double f = frexp(x, &e);
    return __logf((float)f) + (float)e * 0.693147180559945309f;
}

// sqrt(2.0) correctly rounded, the `root2` of the traversal predicates.
#define TD3_ROOT2 1.4142135623730951

// Report a failure into a device status word that the caller zeroed: the first
// reporting thread wins, as tree_d_3d_report of the reference's CUDA kernels
// (K/barnes_hut.cuh:15-20).
__device__ __forceinline__ void td3_report(i64* status, i64 value) {
    atomicCAS(reinterpret_cast<unsigned long long*>(status), 0ULL, (unsigned long long)value);
}

// Two int64 counters scanned together (the 4-way quadrant counts of the build pack two
// 32-bit counts into each word; no count reaches 2^31).
struct td3_i64x2 {
    i64 a, b;
    td3_i64x2() = default;
    __host__ __device__ td3_i64x2(int z) : a(z), b(z) {}
    __host__ __device__ td3_i64x2(i64 x, i64 y) : a(x), b(y) {}
    __host__ __device__ td3_i64x2& operator+=(const td3_i64x2& o) {
        a += o.a;
        b += o.b;
        return *this;
    }
    __host__ __device__ td3_i64x2 operator+(const td3_i64x2& o) const { return td3_i64x2(a + o.a, b + o.b); }
    __host__ __device__ td3_i64x2 operator-(const td3_i64x2& o) const { return td3_i64x2(a - o.a, b - o.b); }
};

// ---------------------------------------------------------------------------------
// Device-wide scans (scan.cu).  Exclusive scan of n items; total (optional) receives the sum.
size_t td3_scan_workspace(i64 n);
int td3_exclusive_scan_i64(const i64* in, i64* out, i64 n, i64* total, void* ws, size_t ws_bytes,
                           cudaStream_t stream);
int td3_exclusive_scan_i32(const int* in, int* out, i64 n, int* total, void* ws, size_t ws_bytes,
                           cudaStream_t stream);
int td3_exclusive_scan_i64x2(const td3_i64x2* in, td3_i64x2* out, i64 n, td3_i64x2* total,
                             void* ws, size_t ws_bytes, cudaStream_t stream);

// The mixed-precision log M2L with its matrix products on the tensor cores, orders up
// to 15 (m2l_tc.cu); arguments as td3_fmm_m2l_mixed, coeff on the host.
int td3_m2l_tensor(const i64* row_start, const int* entry_row, const i64* partners, i64 n_dst,
                   const double* dst_center,
                   const double* dst_half, const double* src_center, const double* src_half,
                   const float2* hat, int order, const double* coeff, double unit,
                   double* local_re, double* local_im, i64* status, cudaStream_t s);

// Stable LSD radix sort of (key, value) pairs by the low `bits` bits of the key
// (scan.cu).  Keys and values are ping-ponged between the in and alt buffers; the
// sorted result is returned in *keys_out / *vals_out (one of the two buffers).
size_t td3_sort_workspace(i64 n);
int td3_radix_sort_u32(unsigned* keys, unsigned* keys_alt, unsigned* vals, unsigned* vals_alt,
                       i64 n, int bits, unsigned** keys_out, unsigned** vals_out, void* ws,
                       size_t ws_bytes, cudaStream_t stream);
