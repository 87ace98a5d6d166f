// Line charges between grounded plates (src/tree_d_3d/strip.py, GroundedStripField):
//   the conformal map zeta = exp(i pi z / L) of the strip 0 < x < L onto the upper
//   half-plane, the charges and their images (-q at conj(zeta)) as one free-space log
//   source set for the FMM / walk / direct sum, the map of the mapped-plane field back
//   to the strip with each charge's own regular term (strip.py:228-246), and the
//   physical-plane softening of close pairs (strip.py:172-201 with the soften_pairs
//   kernel, K/soften_pairs/soften_pairs_pyccel.py:16-52; the probe form strip.py:296-326).
//
// Close pairs are found on the device: sources bucketed by a hash of their cell on a grid
// of the cutoff radius (a stable radix sort of the hashes), every target visits the nine
// cells around its own (each distinct bucket once) and keeps the sources within the
// radius.  A target sums its corrections itself (no atomics), in bucket order.
#include "common.cuh"

namespace {

constexpr double TD3_PI = 3.14159265358979323846;

// zeta of (x, y): exp(-pi y / L) (cos(pi x / L) + i sin(pi x / L)); status 1 + i for a
// point not strictly between the plates.
__global__ void k_strip_map(const double* __restrict__ pos, i64 n, double width,
                            const double* __restrict__ charge, double* __restrict__ out,
                            i64 out_stride, double* __restrict__ out_charge, i64* status) {
    i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double x = pos[i], y = pos[n + i];
    if (!(x > 0.0 && x < width)) td3_report(status, i + 1);
    double a = TD3_PI / width;
    double r = exp(-a * y), s, c;
    sincos(a * x, &s, &c);
    out[i] = r * c;
    out[out_stride + i] = r * s;
    if (charge) {
        // the image: conj(zeta) with -q
        out[n + i] = r * c;
        out[out_stride + n + i] = -(r * s);
        out_charge[i] = charge[i];
        out_charge[n + i] = -charge[i];
    }
}

// Field and potential back in the strip from the mapped-plane sums (raw field E at
// zeta: E_x - i E_y = 2 W'(zeta)):  E_x - i E_y (strip) = (E_x - i E_y)(i pi / L) zeta,
// plus for a charge its own regular term 2 q (i pi / 2L); phi minus 2 q ln(pi |zeta| / L).
__global__ void k_strip_assemble(const double* __restrict__ zeta, i64 zstride, i64 m,
                                 double width, const double* __restrict__ charge,
                                 const double* __restrict__ phi_raw,
                                 const double* __restrict__ field_raw, i64 fstride,
                                 int with_potential, double* __restrict__ phi,
                                 double* __restrict__ field) {
    i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    double zr = zeta[i], zi = zeta[zstride + i];
    double mr = field_raw[i], mi = -field_raw[fstride + i];  // E_x - i E_y
    double a = TD3_PI / width;
    // (mr + i mi) (i a) (zr + i zi)
    double tr = -mi * a, ti = mr * a;
    double cr = tr * zr - ti * zi, ci = tr * zi + ti * zr;
    if (charge) ci += 2.0 * charge[i] * (a / 2.0);
    field[i] = cr;
    field[m + i] = -ci;
    if (!with_potential) {
        phi[i] = 0.0;
    } else if (charge) {
        phi[i] = phi_raw[i] - 2.0 * charge[i] * log(a * sqrt(zr * zr + zi * zi));
    } else {
        phi[i] = phi_raw[i];
    }
}

// ------------------------------------------------------------------ close pairs
__device__ __forceinline__ i64 cell_of(double v, double inv_cell) {
    double c = floor(v * inv_cell);
    c = c < -4.0e15 ? -4.0e15 : (c > 4.0e15 ? 4.0e15 : c);
    return (i64)c;
}

__device__ __forceinline__ unsigned cell_hash(i64 cx, i64 cy, int bits) {
    unsigned long long h = (unsigned long long)cx * 0x9E3779B97F4A7C15ull ^
                           ((unsigned long long)cy + 0x632BE59BD9B4E019ull) * 0xC2B2AE3D27D4EB4Full;
    h ^= h >> 29;
    h *= 0xBF58476D1CE4E5B9ull;
    h ^= h >> 32;
    return (unsigned)(h >> (64 - bits));
}

__global__ void k_cell_keys(const double* __restrict__ pos, i64 n, double inv_cell, int bits,
                            unsigned* __restrict__ keys, unsigned* __restrict__ vals) {
    i64 j = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    keys[j] = cell_hash(cell_of(pos[j], inv_cell), cell_of(pos[n + j], inv_cell), bits);
    vals[j] = (unsigned)j;
}

__device__ __forceinline__ i64 lower_key(const unsigned* __restrict__ keys, i64 n, unsigned h) {
    i64 lo = 0, hi = n;
    while (lo < hi) {
        i64 mid = (lo + hi) >> 1;
        if (keys[mid] < h) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// For target i: the sources within `radius` (not i itself when `same`) replace the bare
// log kernel by the softened one (soften_pairs_pyccel.py:36-52, as the target's share):
// phi += q ln(r^2 / (r^2 + eps^2)), E += q (2 / (r^2 + eps^2) - 2 / r^2) d.  Then the
// results are scaled by `scale` (k_e).  A zero separation reports 1 + i.
__global__ void k_soften(const double* __restrict__ tpos, i64 m, const double* __restrict__ spos,
                         const double* __restrict__ charge, i64 n, int same,
                         const unsigned* __restrict__ keys, const unsigned* __restrict__ vals,
                         double radius, double eps2, int bits, int with_potential, double scale,
                         double* __restrict__ phi, double* __restrict__ field, i64* status) {
    i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    double dphi = 0.0, dfx = 0.0, dfy = 0.0;
    if (keys) {
        double x = tpos[i], y = tpos[m + i];
        double inv_cell = 1.0 / radius, r2max = radius * radius;
        i64 cx = cell_of(x, inv_cell), cy = cell_of(y, inv_cell);
        unsigned seen[9];
        int n_seen = 0;
        for (int oy = -1; oy <= 1; ++oy) {
            for (int ox = -1; ox <= 1; ++ox) {
                unsigned h = cell_hash(cx + ox, cy + oy, bits);
                bool dup = false;
                for (int k = 0; k < n_seen; ++k) dup |= seen[k] == h;
                if (dup) continue;
                seen[n_seen++] = h;
                for (i64 p = lower_key(keys, n, h); p < n && keys[p] == h; ++p) {
                    i64 j = vals[p];
                    if (same && j == i) continue;
                    double dx = x - spos[j], dy = y - spos[n + j];
                    double r2 = dx * dx + dy * dy;
                    if (r2 > r2max) continue;
                    if (r2 == 0.0) {
                        td3_report(status, i + 1);
                        continue;
                    }
                    double soft = r2 + eps2, q = charge[j];
                    if (with_potential) dphi += q * -log(soft / r2);
                    double s = 2.0 / soft - 2.0 / r2;
                    dfx += q * (s * dx);
                    dfy += q * (s * dy);
                }
            }
        }
    }
    phi[i] = with_potential ? scale * (phi[i] + dphi) : 0.0;
    field[i] = scale * (field[i] + dfx);
    field[m + i] = scale * (field[m + i] + dfy);
}

int hash_bits(i64 n) {
    int b = 4;
    while (b < 30 && ((i64)1 << b) < 2 * n) ++b;
    return b;
}

}  // namespace

extern "C" int td3_strip_map(const double* pos, int64_t n, double width, const double* charge,
                             double* sources, double* source_charge, int64_t* status,
                             void* stream) {
    if (n < 0 || !(width > 0.0 && width < INFINITY)) return TD3_EINVAL;
    if (n == 0) return TD3_OK;
    i64 stride = charge ? 2 * n : n;
    k_strip_map<<<td3_blocks(n, 256), 256, 0, td3_stream(stream)>>>(
        pos, n, width, charge, sources, stride, source_charge, status);
    TD3_CHECK_LAUNCH();
    return TD3_OK;
}

extern "C" int td3_strip_assemble(const double* zeta, int64_t zeta_stride, int64_t m,
                                  double width, const double* charge, const double* phi_raw,
                                  const double* field_raw, int64_t field_stride,
                                  int with_potential, double* phi, double* field, void* stream) {
    if (m < 0 || !(width > 0.0 && width < INFINITY)) return TD3_EINVAL;
    if (m == 0) return TD3_OK;
    k_strip_assemble<<<td3_blocks(m, 256), 256, 0, td3_stream(stream)>>>(
        zeta, zeta_stride, m, width, charge, phi_raw, field_raw, field_stride, with_potential, phi,
        field);
    TD3_CHECK_LAUNCH();
    return TD3_OK;
}

extern "C" size_t td3_soften_workspace_size(int64_t n) {
    return 4 * td3_ws_bytes<unsigned>(n) + td3_sort_workspace(n);
}

extern "C" int td3_soften(const double* targets, int64_t m, const double* sources,
                          const double* charge, int64_t n, int same, double radius,
                          double softening, int with_potential, double scale, double* phi,
                          double* field, int64_t* status, void* workspace,
                          size_t workspace_bytes, void* stream) {
    if (m < 0 || n < 0 || !(softening >= 0.0 && softening < INFINITY)) return TD3_EINVAL;
    if (softening > 0.0 && !(radius > 0.0 && radius < INFINITY)) return TD3_EINVAL;
    if (n > 0x7fffffffLL) return TD3_EINVAL;
    if (m == 0) return TD3_OK;
    cudaStream_t s = td3_stream(stream);
    const unsigned *keys = nullptr, *vals = nullptr;
    int bits = hash_bits(n);
    if (softening > 0.0 && n > 0) {
        Workspace w(workspace, workspace_bytes);
        unsigned* k0 = w.take<unsigned>(n);
        unsigned* k1 = w.take<unsigned>(n);
        unsigned* v0 = w.take<unsigned>(n);
        unsigned* v1 = w.take<unsigned>(n);
        if (!v1) return TD3_EWORKSPACE;
        k_cell_keys<<<td3_blocks(n, 256), 256, 0, s>>>(sources, n, 1.0 / radius, bits, k0, v0);
        TD3_CHECK_LAUNCH();
        unsigned *ko, *vo;
        TD3_TRY_RC(td3_radix_sort_u32(k0, k1, v0, v1, n, bits, &ko, &vo, w.base + w.used,
                                      w.size - w.used, s));
        keys = ko;
        vals = vo;
    }
    k_soften<<<td3_blocks(m, 128), 128, 0, s>>>(targets, m, sources, charge, n, same, keys, vals,
                                                radius, softening * softening, bits,
                                                with_potential, scale, phi, field, status);
    TD3_CHECK_LAUNCH();
    return TD3_OK;
}
