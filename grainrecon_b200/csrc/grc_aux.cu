// grc_aux.cu -- preparation, epilogue, distance-map coding and synthetic-data kernels.
#include <cub/cub.cuh>
#include <cuda_runtime.h>
#include <math_constants.h>
#include <stdint.h>

#include "grc_internal.h"

#include <mutex>
#include <vector>

namespace grc {
namespace {

constexpr int kB = 256;

inline int blocks_for(int64_t n, int per = kB) {
    int64_t b = (n + per - 1) / per;
    if (b < 1) b = 1;
    if (b > (1 << 30)) b = 1 << 30;
    return (int)b;
}

// quaternion2U.m:3-28 (no renormalisation: q is used as given).
__global__ void quat_to_u_k(const float *q, int64_t n, double *U) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double q0 = q[4 * i], q1 = q[4 * i + 1], q2 = q[4 * i + 2], q3 = q[4 * i + 3];
        double *u = U + 9 * i;
        u[0] = 2 * (q0 * q0 + q1 * q1) - 1; u[1] = 2 * (q1 * q2 - q0 * q3); u[2] = 2 * (q1 * q3 + q0 * q2);
        u[3] = 2 * (q1 * q2 + q0 * q3); u[4] = 2 * (q0 * q0 + q2 * q2) - 1; u[5] = 2 * (q2 * q3 - q0 * q1);
        u[6] = 2 * (q1 * q3 - q0 * q2); u[7] = 2 * (q2 * q3 + q0 * q1); u[8] = 2 * (q0 * q0 + q3 * q3) - 1;
    }
}

// euler2u.m:5- with angles in degrees (converted as phi*pi/180).
__global__ void euler_to_u_k(const float *e, int64_t n, double *U) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double p1 = (double)e[3 * i] * CUDART_PI / 180, P = (double)e[3 * i + 1] * CUDART_PI / 180,
                     p2 = (double)e[3 * i + 2] * CUDART_PI / 180;
        const double c1 = cos(p1), s1 = sin(p1), c = cos(P), s = sin(P), c2 = cos(p2), s2 = sin(p2);
        double *u = U + 9 * i;
        u[0] = c1 * c2 - s1 * s2 * c; u[1] = -c1 * s2 - s1 * c2 * c; u[2] = s1 * s;
        u[3] = s1 * c2 + c1 * s2 * c; u[4] = -s1 * s2 + c1 * c2 * c; u[5] = -c1 * s;
        u[6] = s2 * s; u[7] = c2 * s; u[8] = c;
    }
}

__global__ void f_to_d_k(const float *a, int64_t n, double *out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (double)a[i];
}

// grow_indexed_region_parallel.m:70-74: pos = ((idx+RVP-1)-Dim/2)*VoxSize+Center, x,y negated for simap.
__global__ void pos_rows_k(const float *rows, int stride, int64_t n, const double *p1, double *vpos) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float *r = rows + (int64_t)stride * i;
        double p[3];
        for (int k = 0; k < 3; ++k) p[k] = (((double)r[k] + p1[k] - 1) - p1[8 + k] / 2) * p1[4] + p1[5 + k];
        if (p1[3] == 1.0) {
            p[0] = -p[0];
            p[1] = -p[1];
        }
        vpos[3 * i] = p[0];
        vpos[3 * i + 1] = p[1];
        vpos[3 * i + 2] = p[2];
    }
}

__global__ void epi_forward_k(const TrialRes *res, int64_t n, float *out, int median) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const TrialRes r = res[i];
        float4 o;
        o.x = (float)r.simu;
        o.y = (float)r.inter;
        o.z = (float)((double)r.inter / (double)r.simu);  // Nr_intersect/Nr_simu, NaN for 0/0
        o.w = median ? (float)r.median : CUDART_NAN_F;    // no median in completeness-only calls
        reinterpret_cast<float4 *>(out)[i] = o;
    }
}

// Accept rule of grow_indexed_region_parallel.m:78-88 without the Ninter clause.
__global__ void epi_grow_k(const TrialRes *res, const float *rows6, int64_t m, const double *p1, float *out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
        const TrialRes r = res[i];
        const float *row = rows6 + 6 * i;
        const double C = (double)r.inter / (double)r.simu;
        const double I = row[3], mask = row[4], dmed = row[5];
        const double lim = fmin(dmed, p1[13]);
        const bool cand = mask > 0 && C > I && r.median <= lim;
        const bool flag = cand && C >= p1[11] * (1 - p1[12]);
        float *w = out + 7 * i;
        w[0] = row[0];
        w[1] = row[1];
        w[2] = row[2];
        w[3] = (float)r.simu;
        w[4] = (float)r.inter;
        w[5] = (float)r.median;
        w[6] = flag ? 1.0f : 0.0f;
    }
}

__global__ void csr_counts_k(const float *rows5, int64_t m, int64_t *counts) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t first = (int64_t)rows5[5 * i + 3], last = (int64_t)rows5[5 * i + 4];
        counts[i] = last >= first ? last - first + 1 : 0;
    }
}

__global__ void csr_fill_k(const float *rows5, int64_t m, const int64_t *off, const float *id_neigb, int64_t n_neigb,
                           int64_t n_grain, longlong4 *items, int32_t *trial_orient, int32_t *trial_voxel, int *bad) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t first = (int64_t)rows5[5 * i + 3], last = (int64_t)rows5[5 * i + 4];
        const int64_t o = off[i];
        int64_t cnt = last >= first ? last - first + 1 : 0;
        if (cnt > 0 && (first < 1 || last > n_neigb)) {
            atomicOr(bad, 1);
            cnt = 0;
        }
        for (int64_t j = 0; j < cnt; ++j) {
            int64_t gid = (int64_t)id_neigb[first - 1 + j];
            if (gid < 1 || gid > n_grain) {
                atomicOr(bad, 2);
                gid = 1;
            }
            trial_orient[o + j] = (int32_t)(gid - 1);
            trial_voxel[o + j] = (int32_t)i;
        }
        items[i] = make_longlong4(i, o, o + cnt, 0);
    }
}

// Argmax over each voxel's candidates with MATLAB max semantics (first max, NaN ignored).
__global__ void epi_compete_k(const TrialRes *res, const longlong4 *items, const int32_t *trial_orient, int64_t m,
                              const float *euler, float *out, float *trial_out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
        const longlong4 it = items[i];
        float *w = out + 8 * i;
        w[0] = (float)(i + 1);
        for (int k = 1; k < 8; ++k) w[k] = 0.f;
        w[7] = 2000.f;
        int64_t best = -1;
        double bestC = CUDART_NAN;
        for (int64_t t = it.y; t < it.z; ++t) {
            const TrialRes r = res[t];
            const double C = (double)r.inter / (double)r.simu;
            if (best < 0 || (!isnan(C) && (isnan(bestC) || C > bestC))) {
                best = t;
                bestC = C;
            }
            if (trial_out) {
                float4 o;
                o.x = (float)r.simu;
                o.y = (float)r.inter;
                o.z = (float)C;
                o.w = (float)r.median;
                reinterpret_cast<float4 *>(trial_out)[t] = o;
            }
        }
        if (best >= 0) {
            const int32_t gi = trial_orient[best];
            const TrialRes r = res[best];
            w[1] = euler[3 * gi];
            w[2] = euler[3 * gi + 1];
            w[3] = euler[3 * gi + 2];
            w[4] = (float)(gi + 1);
            w[5] = (float)bestC;
            w[6] = (float)r.inter;
            w[7] = (float)r.median;
        }
    }
}

// grow_unindexed_compete_comp_cuda.m:51-64 on device: write each voxel's winner into the
// sample maps (MATLAB column-major volumes, 1-based voxel indices in rows5).
__global__ void apply_compete_k(const float *out8, const float *rows5, int64_t m, int64_t d1, int64_t d2,
                                int64_t d3, float *comp, float *gid, float *dmed, float *ninter, float *visit) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t x = (int64_t)rows5[5 * i] - 1, y = (int64_t)rows5[5 * i + 1] - 1, z = (int64_t)rows5[5 * i + 2] - 1;
        if (x < 0 || y < 0 || z < 0 || x >= d1 || y >= d2 || z >= d3) continue;
        const int64_t k = x + d1 * (y + d2 * z);
        const float *o = out8 + 8 * i;
        if (comp) comp[k] = o[5];
        if (gid) gid[k] = o[4];
        if (dmed) dmed[k] = o[7];
        if (ninter) ninter[k] = o[6];
        if (visit) visit[k] = 0.5f;
    }
}

// ---- distance-map rank coding --------------------------------------------------
// Each float maps to an order-preserving 32-bit key; a 2^32-bit presence bitmap
// plus a prefix popcount gives every value its rank among the distinct values.

__device__ __forceinline__ uint32_t ordered_key(float v) {
    if (v == 0.0f) v = 0.0f;  // -0 and +0 are the same value
    const uint32_t b = __float_as_uint(v);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

__device__ __forceinline__ float key_value(uint32_t k) {
    const uint32_t b = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
    return __uint_as_float(b);
}

__global__ void mark_values_k(const float *map, int64_t n, uint32_t *bitmap, int *bad) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float v = map[i];
        if (isnan(v)) {
            atomicOr(bad, 1);
            continue;
        }
        const uint32_t k = ordered_key(v);
        const uint32_t bit = 1u << (k & 31);
        if (!(bitmap[k >> 5] & bit)) atomicOr(&bitmap[k >> 5], bit);
    }
}

__global__ void popc_k(const uint32_t *bitmap, int64_t nw, uint32_t *cnt) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nw; i += (int64_t)gridDim.x * blockDim.x)
        cnt[i] = __popc(bitmap[i]);
}

__global__ void values_k(const uint32_t *bitmap, const uint32_t *prefix, int64_t nw, float *vals) {
    for (int64_t w = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; w < nw; w += (int64_t)gridDim.x * blockDim.x) {
        uint32_t bits = bitmap[w];
        uint32_t r = prefix[w];
        while (bits) {
            const int b = __ffs(bits) - 1;
            bits &= bits - 1;
            vals[r++] = key_value(((uint32_t)w << 5) | (uint32_t)b);
        }
    }
}

template <typename CodeT>
__global__ void codes_k(const float *map, int64_t n, const uint32_t *bitmap, const uint32_t *prefix, CodeT *codes,
                        uint8_t *codes8) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t k = ordered_key(map[i]);
        const uint32_t w = k >> 5, b = k & 31;
        const uint32_t c = prefix[w] + __popc(bitmap[w] & ((1u << b) - 1u));
        codes[i] = (CodeT)c;
        codes8[i] = (uint8_t)(c < 255u ? c : 255u);
    }
}

// ---- exact EDT (bwdist semantics) ------------------------------------------------
// Pass 1: along detz (contiguous) the squared distance to the nearest marked pixel
// of the same line (two sweeps).  Pass 2: along dety, D(y) = min_y' g(y') + (y-y')^2
// by an outward search that stops once (y-y')^2 exceeds the best value.
__global__ void edt_lines_k(const uint8_t *mask, int64_t nz, int64_t nlines, float *g) {
    for (int64_t line = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; line < nlines;
         line += (int64_t)gridDim.x * blockDim.x) {
        const uint8_t *m = mask + line * nz;
        float *o = g + line * nz;
        int64_t last = -1;
        for (int64_t z = 0; z < nz; ++z) {
            if (m[z]) last = z;
            o[z] = last < 0 ? CUDART_INF_F : (float)((z - last) * (z - last));
        }
        last = -1;
        for (int64_t z = nz - 1; z >= 0; --z) {
            if (m[z]) last = z;
            if (last >= 0) {
                const float d = (float)((last - z) * (last - z));
                if (d < o[z]) o[z] = d;
            }
        }
    }
}

__global__ void edt_cols_k(const float *g, int64_t nz, int64_t ny, int64_t nrot, float *map) {
    const int64_t n = nz * ny * nrot;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t z = i % nz;
        const int64_t y = (i / nz) % ny;
        const int64_t base = i - y * nz;  // (iw, 0, z)
        float best = g[i];
        for (int64_t d = 1; (float)(d * d) < best && (y - d >= 0 || y + d < ny); ++d) {
            const float dd = (float)(d * d);
            if (y - d >= 0) {
                const float c = g[base + (y - d) * nz] + dd;
                if (c < best) best = c;
            }
            if (y + d < ny) {
                const float c = g[base + (y + d) * nz] + dd;
                if (c < best) best = c;
            }
        }
        map[i] = isinf(best) ? CUDART_INF_F : sqrtf(best);
        (void)z;
    }
}

}  // namespace

namespace {
struct OccEntry {
    int device;
    const void *fn;
    size_t smem;
    int per_sm;
};
struct SmemEntry {
    int device;
    const void *fn;
    size_t allowed;
};
std::mutex g_launch_mu;
std::vector<OccEntry> g_occ;
std::vector<SmemEntry> g_smem;

// caller holds g_launch_mu
cudaError_t allow_smem_locked(int dev, const void *fn, size_t smem) {
    for (SmemEntry &e : g_smem)
        if (e.device == dev && e.fn == fn) {
            if (e.allowed >= smem) return cudaSuccess;
            const cudaError_t r = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (r == cudaSuccess) e.allowed = smem;
            return r;
        }
    const cudaError_t r = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (r == cudaSuccess) g_smem.push_back({dev, fn, smem});
    return r;
}
}  // namespace

cudaError_t allow_smem(const void *fn, size_t smem) {
    int dev = 0;
    cudaError_t r = cudaGetDevice(&dev);
    if (r != cudaSuccess) return r;
    std::lock_guard<std::mutex> g(g_launch_mu);
    return allow_smem_locked(dev, fn, smem);
}

cudaError_t occupancy_for(const void *fn, size_t smem, int *per_sm) {
    int dev = 0;
    cudaError_t r = cudaGetDevice(&dev);
    if (r != cudaSuccess) return r;
    std::lock_guard<std::mutex> g(g_launch_mu);
    for (const OccEntry &e : g_occ)
        if (e.device == dev && e.fn == fn && e.smem == smem) {
            *per_sm = e.per_sm;
            return cudaSuccess;
        }
    r = allow_smem_locked(dev, fn, smem);
    if (r != cudaSuccess) return r;
    int n = 0;
    r = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, kThreads, smem);
    if (r != cudaSuccess) return r;
    g_occ.push_back({dev, fn, smem, n});
    *per_sm = n;
    return cudaSuccess;
}

cudaError_t launch_quat_to_u(const float *q, int64_t n, double *U, cudaStream_t s) {
    quat_to_u_k<<<blocks_for(n), kB, 0, s>>>(q, n, U);
    return cudaGetLastError();
}
cudaError_t launch_euler_to_u(const float *e, int64_t n, double *U, cudaStream_t s) {
    euler_to_u_k<<<blocks_for(n), kB, 0, s>>>(e, n, U);
    return cudaGetLastError();
}
cudaError_t launch_f9_to_u(const float *u9, int64_t n, double *U, cudaStream_t s) {
    f_to_d_k<<<blocks_for(9 * n), kB, 0, s>>>(u9, 9 * n, U);
    return cudaGetLastError();
}
cudaError_t launch_pos_f3(const float *p, int64_t n, double *vpos, cudaStream_t s) {
    f_to_d_k<<<blocks_for(3 * n), kB, 0, s>>>(p, 3 * n, vpos);
    return cudaGetLastError();
}
cudaError_t launch_pos_rows(const float *rows, int stride, int64_t n, const double *p1, double *vpos,
                            cudaStream_t s) {
    pos_rows_k<<<blocks_for(n), kB, 0, s>>>(rows, stride, n, p1, vpos);
    return cudaGetLastError();
}
cudaError_t launch_epi_forward(const TrialRes *res, int64_t n, float *out4, bool median, cudaStream_t s) {
    epi_forward_k<<<blocks_for(n), kB, 0, s>>>(res, n, out4, median ? 1 : 0);
    return cudaGetLastError();
}
cudaError_t launch_epi_grow(const TrialRes *res, const float *rows6, int64_t m, const double *p1, float *out7,
                            cudaStream_t s) {
    epi_grow_k<<<blocks_for(m), kB, 0, s>>>(res, rows6, m, p1, out7);
    return cudaGetLastError();
}
cudaError_t launch_csr_counts(const float *rows5, int64_t m, int64_t *counts, cudaStream_t s) {
    csr_counts_k<<<blocks_for(m), kB, 0, s>>>(rows5, m, counts);
    return cudaGetLastError();
}
cudaError_t launch_csr_fill(const float *rows5, int64_t m, const int64_t *offsets, const float *id_neigb,
                            int64_t n_neigb, int64_t n_grain, longlong4 *items, int32_t *trial_orient,
                            int32_t *trial_voxel, int *bad, cudaStream_t s) {
    csr_fill_k<<<blocks_for(m), kB, 0, s>>>(rows5, m, offsets, id_neigb, n_neigb, n_grain, items, trial_orient,
                                            trial_voxel, bad);
    return cudaGetLastError();
}
cudaError_t launch_epi_compete(const TrialRes *res, const longlong4 *items, const int32_t *trial_orient, int64_t m,
                               const float *euler, float *out8, float *trial_out4, cudaStream_t s) {
    epi_compete_k<<<blocks_for(m), kB, 0, s>>>(res, items, trial_orient, m, euler, out8, trial_out4);
    return cudaGetLastError();
}

cudaError_t launch_apply_compete(const float *out8, const float *rows5, int64_t m, const int64_t *dims, float *comp,
                                 float *gid, float *dmed, float *ninter, float *visit, cudaStream_t s) {
    apply_compete_k<<<blocks_for(m), kB, 0, s>>>(out8, rows5, m, dims[0], dims[1], dims[2], comp, gid, dmed, ninter,
                                                 visit);
    return cudaGetLastError();
}

cudaError_t encode_map(const float *d_map, int64_t n, cudaStream_t s, MapCodes *out, int *bad_nan) {
    const int64_t nw = int64_t(1) << 27;  // 2^32 bits
    uint32_t *bitmap = nullptr, *cnt = nullptr, *prefix = nullptr;
    int *d_bad = nullptr;
    void *tmp = nullptr;
    size_t tmp_bytes = 0;
    cudaError_t e;
    out->codes = nullptr;
    out->codes8 = nullptr;
    out->vals = nullptr;
#define CK(x)                    \
    do {                         \
        e = (x);                 \
        if (e != cudaSuccess) {  \
            goto done;           \
        }                        \
    } while (0)
    CK(cudaMalloc(&bitmap, nw * 4));
    CK(cudaMalloc(&cnt, nw * 4));
    CK(cudaMalloc(&prefix, nw * 4));
    CK(cudaMalloc(&d_bad, sizeof(int)));
    CK(cudaMemsetAsync(bitmap, 0, nw * 4, s));
    CK(cudaMemsetAsync(d_bad, 0, sizeof(int), s));
    mark_values_k<<<blocks_for(n, kB * 8), kB, 0, s>>>(d_map, n, bitmap, d_bad);
    CK(cudaGetLastError());
    popc_k<<<blocks_for(nw), kB, 0, s>>>(bitmap, nw, cnt);
    CK(cudaGetLastError());
    CK(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, cnt, prefix, (int)nw, s));
    CK(cudaMalloc(&tmp, tmp_bytes));
    CK(cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, cnt, prefix, (int)nw, s));
    {
        uint32_t last_prefix = 0, last_cnt = 0;
        int hbad = 0;
        CK(cudaMemcpyAsync(&last_prefix, prefix + nw - 1, 4, cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(&last_cnt, cnt + nw - 1, 4, cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(&hbad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        *bad_nan = hbad;
        if (hbad) goto done;
        const int64_t nd = (int64_t)last_prefix + last_cnt;
        out->n_distinct = nd;
        int bits = 0;
        while (bits < 32 && (int64_t(1) << bits) < nd) ++bits;
        CK(cudaMalloc(&out->vals, sizeof(float) * (nd > 0 ? nd : 1)));
        values_k<<<blocks_for(nw), kB, 0, s>>>(bitmap, prefix, nw, out->vals);
        CK(cudaGetLastError());
        CK(cudaMalloc(&out->codes8, sizeof(uint8_t) * (n > 0 ? n : 1)));
        out->code_bits = bits;
        if (nd <= 65536) {
            CK(cudaMalloc(&out->codes, sizeof(uint16_t) * (n > 0 ? n : 1)));
            codes_k<uint16_t><<<blocks_for(n, kB * 8), kB, 0, s>>>(d_map, n, bitmap, prefix, (uint16_t *)out->codes,
                                                                  out->codes8);
        } else {
            CK(cudaMalloc(&out->codes, sizeof(uint32_t) * (n > 0 ? n : 1)));
            codes_k<uint32_t><<<blocks_for(n, kB * 8), kB, 0, s>>>(d_map, n, bitmap, prefix, (uint32_t *)out->codes,
                                                                  out->codes8);
        }
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(s));
    }
done:
#undef CK
    cudaFree(bitmap);
    cudaFree(cnt);
    cudaFree(prefix);
    cudaFree(d_bad);
    cudaFree(tmp);
    if (e != cudaSuccess || *bad_nan) {
        cudaFree(out->codes);
        cudaFree(out->codes8);
        cudaFree(out->vals);
        out->codes = nullptr;
        out->codes8 = nullptr;
        out->vals = nullptr;
    }
    return e;
}

cudaError_t launch_edt(const uint8_t *mask, int64_t nz, int64_t ny, int64_t nrot, float *map, cudaStream_t s) {
    float *g = nullptr;
    cudaError_t e = cudaMalloc(&g, sizeof(float) * nz * ny * nrot);
    if (e != cudaSuccess) return e;
    edt_lines_k<<<blocks_for(ny * nrot, 128), 128, 0, s>>>(mask, nz, ny * nrot, g);
    edt_cols_k<<<blocks_for(nz * ny * nrot, kB * 4), kB, 0, s>>>(g, nz, ny, nrot, map);
    e = cudaGetLastError();
    cudaError_t e2 = cudaStreamSynchronize(s);
    cudaFree(g);
    return e != cudaSuccess ? e : e2;
}

}  // namespace grc
