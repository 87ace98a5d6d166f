// Exact all-pairs sums: direct_field of both kernels and the Coulomb pair energy.
//
// One thread per target; the sources stream through shared memory in tiles of
// DIRECT_THREADS (x, y, q staged once per block and read as warp broadcasts).  When
// the targets alone cannot fill the GPU (few targets, many sources), the sources are
// split into chunks along gridDim.y and each chunk writes partial sums to the
// workspace, reduced afterwards in a fixed order (deterministic results).
#include <mutex>

#include "common.cuh"

namespace {

constexpr int DIRECT_THREADS = 256;
constexpr int SM_COUNT_B200 = 148;

template <int KERNEL, bool POT, bool PARTIAL>
__global__ void __launch_bounds__(DIRECT_THREADS)
k_direct(const double* __restrict__ targets, i64 m, const i64* __restrict__ exclude,
         const double* __restrict__ pos, const double* __restrict__ charge, i64 n, i64 chunk,
         double eps2, double* __restrict__ phi, double* __restrict__ field,
         double* __restrict__ partial, i64* status) {
    __shared__ double sx[DIRECT_THREADS], sy[DIRECT_THREADS], sq[DIRECT_THREADS];
    i64 i = (i64)blockIdx.x * DIRECT_THREADS + threadIdx.x;
    bool live = i < m;
    double tx = live ? targets[i] : 0.0;
    double ty = live ? targets[m + i] : 0.0;
    i64 skip = live ? exclude[i] : -1;
    double p = 0.0, ex = 0.0, ey = 0.0;
    bool bad = false;
    i64 j0 = (i64)blockIdx.y * chunk;
    i64 j1 = j0 + chunk < n ? j0 + chunk : n;
    for (i64 base = j0; base < j1; base += DIRECT_THREADS) {
        i64 j = base + threadIdx.x;
        if (j < j1) {
            sx[threadIdx.x] = pos[j];
            sy[threadIdx.x] = pos[n + j];
            sq[threadIdx.x] = charge[j];
        }
        __syncthreads();
        int count = (int)(j1 - base < DIRECT_THREADS ? j1 - base : DIRECT_THREADS);
        for (int t = 0; t < count; ++t) {
            double c = sq[t];
            if (c == 0.0) continue;  // uniform across the block
            double dx = tx - sx[t];
            double dy = ty - sy[t];
            double r2 = dx * dx + dy * dy + eps2;
            bool own = (base + t) == skip;
            double cb = own ? 0.0 : c;
            r2 = own ? 1.0 : r2;
            bad |= (r2 == 0.0);
            if (KERNEL == TD3_KERNEL_COULOMB) {
                double inv_r = rsqrt(r2);
                double inv_r3 = inv_r * inv_r * inv_r;
                p += cb * inv_r;
                ex += cb * inv_r3 * dx;
                ey += cb * inv_r3 * dy;
            } else {
                if (POT) p -= cb * log(r2);
                double f = 2.0 * cb / r2;
                ex += f * dx;
                ey += f * dy;
            }
        }
        __syncthreads();
    }
    if (!live) return;
    if (bad) td3_report(status, i + 1);
    if (!POT) p = 0.0;
    if (PARTIAL) {
        i64 y = blockIdx.y;
        partial[(3 * y) * m + i] = p;
        partial[(3 * y + 1) * m + i] = ex;
        partial[(3 * y + 2) * m + i] = ey;
    } else {
        phi[i] = p;
        field[i] = ex;
        field[m + i] = ey;
    }
}

__global__ void k_direct_reduce(const double* __restrict__ partial, i64 m, int chunks,
                                double* __restrict__ phi, double* __restrict__ field) {
    i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    double p = 0.0, ex = 0.0, ey = 0.0;
    for (int y = 0; y < chunks; ++y) {
        p += partial[(3 * (i64)y) * m + i];
        ex += partial[(3 * (i64)y + 1) * m + i];
        ey += partial[(3 * (i64)y + 2) * m + i];
    }
    phi[i] = p;
    field[i] = ex;
    field[m + i] = ey;
}

// Source chunks so that (target blocks x chunks) fills the GPU a few times over,
// with at least 2048 sources per chunk.
int direct_chunks(i64 m, i64 n) {
    i64 bx = (m + DIRECT_THREADS - 1) / DIRECT_THREADS;
    i64 want = (4 * SM_COUNT_B200 + bx - 1) / bx;
    i64 most = (n + 2047) / 2048;
    i64 c = want < most ? want : most;
    if (c > 256) c = 256;
    return (int)(c < 1 ? 1 : c);
}

template <int KERNEL, bool POT>
int launch_direct(const double* targets, i64 m, const i64* exclude, const double* pos,
                  const double* charge, i64 n, double eps2, double* phi, double* field,
                  i64* status, double* partial, int chunks, cudaStream_t stream) {
    i64 chunk = (n + chunks - 1) / chunks;
    dim3 grid(td3_blocks(m, DIRECT_THREADS), chunks);
    if (chunks > 1) {
        k_direct<KERNEL, POT, true><<<grid, DIRECT_THREADS, 0, stream>>>(
            targets, m, exclude, pos, charge, n, chunk, eps2, phi, field, partial, status);
        k_direct_reduce<<<td3_blocks(m, 256), 256, 0, stream>>>(partial, m, chunks, phi, field);
    } else {
        k_direct<KERNEL, POT, false><<<grid, DIRECT_THREADS, 0, stream>>>(
            targets, m, exclude, pos, charge, n, chunk, eps2, phi, field, partial, status);
    }
    TD3_CHECK_LAUNCH();
    return TD3_OK;
}

// ------------------------------------------------------------------ pair energy
constexpr int ENERGY_THREADS = 256;

// Row i sums q_j / sqrt(r^2 + eps^2) over j > i; each block writes q_i-weighted
// row sums of its rows to partial[block] (reduced in block order afterwards).
__global__ void __launch_bounds__(ENERGY_THREADS)
k_pair_energy(const double* __restrict__ pos, const double* __restrict__ charge, i64 n,
              double eps2, double* __restrict__ partial, i64* status) {
    __shared__ double sx[ENERGY_THREADS], sy[ENERGY_THREADS], sq[ENERGY_THREADS];
    __shared__ double warp_sum[ENERGY_THREADS / 32];
    i64 i = (i64)blockIdx.x * ENERGY_THREADS + threadIdx.x;
    bool live = i < n;
    double xi = live ? pos[i] : 0.0, yi = live ? pos[n + i] : 0.0;
    double qi = live ? charge[i] : 0.0;
    double row = 0.0;
    bool bad = false;
    i64 first = (i64)blockIdx.x * ENERGY_THREADS;
    for (i64 base = first; base < n; base += ENERGY_THREADS) {
        i64 j = base + threadIdx.x;
        if (j < n) {
            sx[threadIdx.x] = pos[j];
            sy[threadIdx.x] = pos[n + j];
            sq[threadIdx.x] = charge[j];
        }
        __syncthreads();
        int count = (int)(n - base < ENERGY_THREADS ? n - base : ENERGY_THREADS);
        for (int t = 0; t < count; ++t) {
            double cj = sq[t];
            if (cj == 0.0 || base + t <= i) continue;
            double dx = xi - sx[t], dy = yi - sy[t];
            double r2 = dx * dx + dy * dy + eps2;
            bad |= (r2 == 0.0 && qi != 0.0);
            row += cj * rsqrt(r2);
        }
        __syncthreads();
    }
    if (bad) td3_report(status, 1);
    double v = (live && qi != 0.0) ? qi * row : 0.0;
    for (int d = 16; d > 0; d >>= 1) v += __shfl_down_sync(0xffffffffu, v, d);
    if ((threadIdx.x & 31) == 0) warp_sum[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < ENERGY_THREADS / 32; ++w) s += warp_sum[w];
        partial[blockIdx.x] = s;
    }
}

__global__ void k_sum_into(const double* __restrict__ partial, i64 count, double* out) {
    __shared__ double buf[256];
    double s = 0.0;
    for (i64 k = threadIdx.x; k < count; k += 256) s += partial[k];
    buf[threadIdx.x] = s;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) buf[threadIdx.x] += buf[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[0] += buf[0];
}

}  // namespace

extern "C" size_t td3_direct_sum_workspace_size(int64_t n_targets, int64_t n_sources) {
    int chunks = direct_chunks(n_targets, n_sources);
    return chunks > 1 ? td3_ws_bytes<double>(3 * (i64)chunks * n_targets) : 256;
}

extern "C" int td3_direct_sum(int kernel, const double* targets, int64_t m, const int64_t* exclude,
                              const double* pos, const double* charge, int64_t n,
                              double softening, int with_potential, double* phi, double* field,
                              int64_t* status, void* workspace, size_t workspace_bytes,
                              void* stream) {
    if (m < 0 || n < 0 || (kernel != TD3_KERNEL_COULOMB && kernel != TD3_KERNEL_LOG))
        return TD3_EINVAL;
    cudaStream_t s = td3_stream(stream);
    if (m == 0) return TD3_OK;
    if (n == 0) {
        TD3_TRY(cudaMemsetAsync(phi, 0, sizeof(double) * m, s));
        TD3_TRY(cudaMemsetAsync(field, 0, sizeof(double) * 2 * m, s));
        return TD3_OK;
    }
    int chunks = direct_chunks(m, n);
    if (chunks > 1 && workspace_bytes < (size_t)3 * chunks * m * sizeof(double))
        return TD3_EWORKSPACE;
    double* partial = static_cast<double*>(workspace);
    double eps2 = softening * softening;
    bool pot = with_potential != 0;
    if (kernel == TD3_KERNEL_COULOMB)
        return pot ? launch_direct<TD3_KERNEL_COULOMB, true>(targets, m, exclude, pos, charge, n, eps2,
                                                              phi, field, status, partial, chunks, s)
                   : launch_direct<TD3_KERNEL_COULOMB, false>(targets, m, exclude, pos, charge, n,
                                                               eps2, phi, field, status, partial,
                                                               chunks, s);
    return pot ? launch_direct<TD3_KERNEL_LOG, true>(targets, m, exclude, pos, charge, n, eps2, phi,
                                                      field, status, partial, chunks, s)
               : launch_direct<TD3_KERNEL_LOG, false>(targets, m, exclude, pos, charge, n, eps2, phi,
                                                       field, status, partial, chunks, s);
}

extern "C" size_t td3_pair_energy_workspace_size(int64_t n) {
    return td3_ws_bytes<double>((n + ENERGY_THREADS - 1) / ENERGY_THREADS);
}

extern "C" int td3_pair_energy(const double* pos, const double* charge, int64_t n,
                               double softening, double* energy, int64_t* status,
                               void* workspace, size_t workspace_bytes, void* stream) {
    if (n < 0) return TD3_EINVAL;
    if (n < 2) return TD3_OK;
    i64 blocks = (n + ENERGY_THREADS - 1) / ENERGY_THREADS;
    if (workspace_bytes < (size_t)blocks * sizeof(double)) return TD3_EWORKSPACE;
    cudaStream_t s = td3_stream(stream);
    double* partial = static_cast<double*>(workspace);
    k_pair_energy<<<(unsigned)blocks, ENERGY_THREADS, 0, s>>>(pos, charge, n, softening * softening,
                                                               partial, status);
    k_sum_into<<<1, 256, 0, s>>>(partial, blocks, energy);
    TD3_CHECK_LAUNCH();
    return TD3_OK;
}

// ------------------------------------------------------------------ without allocation
//
// td3_direct_sum_noalloc is td3_direct_sum for callers that cannot allocate device
// memory: code running inside a host application that owns all device memory and
// hands the solver only its inputs and outputs (a plugin with a fixed memory budget,
// a control loop where an allocation could block).  Its scratch -- the partial sums of
// the source chunks -- lives in the array below, a fixed part of every device that
// loads the library, kept until the process exits.  The array holds the partial sums
// of any call with at most TD3_DIRECT_NOALLOC_MAX_TARGETS targets (any number of
// sources): 3 x chunks x targets doubles, at most 605,184 (4.6 MiB) for the chunk
// counts that td3_direct_sum chooses.
namespace {

constexpr i64 NOALLOC_SCRATCH_DOUBLES = 605184;
constexpr int NOALLOC_MAX_DEVICES = 64;

static __device__ __align__(256) double g_direct_scratch[NOALLOC_SCRATCH_DOUBLES];

std::mutex g_scratch_mutex;
double* g_scratch_address[NOALLOC_MAX_DEVICES] = {};

// The device address of g_direct_scratch on the current device, looked up once per
// device.  In host code the array's name is only a host-side stand-in, so the address
// must come from cudaGetSymbolAddress with that device current.  The address is kept
// for the life of the process; a cudaDeviceReset (which destroys the context that
// holds the array) would leave it stale, so callers of this entry point must not
// reset the device between calls (stated in the header).
int noalloc_scratch(double** out) {
    int dev = 0;
    TD3_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return TD3_EINVAL;
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_address[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_direct_scratch);
        if (e != cudaSuccess) return td3_cuda_error(e);
        g_scratch_address[dev] = static_cast<double*>(p);
    }
    *out = g_scratch_address[dev];
    return TD3_OK;
}

}  // namespace

extern "C" int td3_direct_sum_noalloc(int kernel, const double* targets, int64_t m,
                                      const int64_t* exclude, const double* pos,
                                      const double* charge, int64_t n, double softening,
                                      int with_potential, double* phi, double* field,
                                      int64_t* status, void* stream) {
    if (m < 0 || n < 0 || (kernel != TD3_KERNEL_COULOMB && kernel != TD3_KERNEL_LOG))
        return TD3_EINVAL;
    if (m > TD3_DIRECT_NOALLOC_MAX_TARGETS) {
        td3_set_error("td3_direct_sum_noalloc: more targets than its fixed scratch holds "
                      "(TD3_DIRECT_NOALLOC_MAX_TARGETS); use td3_direct_sum with a workspace");
        return TD3_ETOOLARGE;
    }
    double* scratch = nullptr;
    TD3_TRY_RC(noalloc_scratch(&scratch));
    cudaStream_t s = td3_stream(stream);
    if (m == 0) return TD3_OK;
    if (n == 0) {
        TD3_TRY(cudaMemsetAsync(phi, 0, sizeof(double) * m, s));
        TD3_TRY(cudaMemsetAsync(field, 0, sizeof(double) * 2 * m, s));
        return TD3_OK;
    }
    int chunks = direct_chunks(m, n);
    if (chunks > 1 && (i64)3 * chunks * m > NOALLOC_SCRATCH_DOUBLES) {
        td3_set_error("td3_direct_sum_noalloc: the partial sums exceed the fixed scratch");
        return TD3_ETOOLARGE;
    }
    // every partial slot the reduction reads is written by the chunk pass first, so
    // the scratch needs no clearing between calls
    double eps2 = softening * softening;
    bool pot = with_potential != 0;
    if (kernel == TD3_KERNEL_COULOMB)
        return pot ? launch_direct<TD3_KERNEL_COULOMB, true>(targets, m, exclude, pos, charge, n, eps2,
                                                              phi, field, status, scratch, chunks, s)
                   : launch_direct<TD3_KERNEL_COULOMB, false>(targets, m, exclude, pos, charge, n,
                                                               eps2, phi, field, status, scratch,
                                                               chunks, s);
    return pot ? launch_direct<TD3_KERNEL_LOG, true>(targets, m, exclude, pos, charge, n, eps2, phi,
                                                      field, status, scratch, chunks, s)
               : launch_direct<TD3_KERNEL_LOG, false>(targets, m, exclude, pos, charge, n, eps2, phi,
                                                       field, status, scratch, chunks, s);
}
