// grc_select.cu -- ordering work of the seeding stage on the device.
//
//   * top_rows_k: sortrows(Output, 3, 'descend') followed by the first n_top rows
//     (GrainMapping_engine_gpu_comp.m:103-111, fit_OR_constrain_with_local_comp_cuda.m:112):
//     per group of completeness values, a radix select of the n_top-th key, the rows above it
//     plus the first rows equal to it, then a bitonic sort of those few rows in shared memory.
//     Order: NaN first (MATLAB's descending sort), then larger values, equal values in their
//     original order (sortrows is stable).
//   * local_grid_k: ori_local_sampling(q, nr, gridsize) (ori_local_sampling.m:12-34): the centre
//     row and the (nr+1)^3 grid rows [sqrt(1-(b^2+c^2+d^2)) b c d], in unique(q, 'rows') order
//     (ascending by q0, b, c, d; a row equal to another stays next to it in the original order).
// Every arithmetic step is rounded separately (no contraction), as the host restatement.
#include <cuda_runtime.h>
#include <math_constants.h>
#include <stdint.h>

#include "grc_internal.h"

namespace grc {
namespace {

constexpr unsigned kAll = 0xffffffffu;
constexpr int kSelThreads = 1024;
constexpr int kSelMaxTop = 4096;  // rows one group may select (shared-memory sort)

// Descending-order key of a completeness value: NaN above everything, then larger values.
__device__ __forceinline__ uint32_t desc_key(float c) {
    if (isnan(c)) return 0xffffffffu;
    if (c == 0.0f) c = 0.0f;  // -0 and +0 compare equal
    const uint32_t u = __float_as_uint(c);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

// Completeness of row i: a float column (vals, stride floats apart) or, when vals is NULL, the
// trial results (Nr_intersect / Nr_simu rounded to float, as the output's column 3).
__device__ __forceinline__ uint32_t val_key(const float *vals, const TrialRes *res, int64_t stride, int64_t i) {
    if (vals) return desc_key(__ldg(vals + i * stride));
    const TrialRes r = res[i];
    return desc_key((float)((double)r.inter / (double)r.simu));
}

// Block-wide exclusive prefix of one flag per thread (1024 threads) plus the block total.
__device__ __forceinline__ int block_prefix(bool f, int *s_warp, int *total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned m = __ballot_sync(kAll, f);
    if (lane == 0) s_warp[warp] = __popc(m);
    __syncthreads();
    if (warp == 0) {
        const int v = s_warp[lane];
        int incl = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(kAll, incl, o);
            if (lane >= o) incl += y;
        }
        s_warp[lane] = incl - v;
        if (lane == 31) s_warp[32] = incl;
    }
    __syncthreads();
    const int r = s_warp[warp] + __popc(m & ((1u << lane) - 1u));
    *total = s_warp[32];
    __syncthreads();
    return r;
}

// One block per group: idx[g*n_top + k] = row of rank k.  Rows with stride `stride` floats.
__global__ void __launch_bounds__(kSelThreads) top_rows_k(const float *vals, const TrialRes *res, int64_t stride,
                                                          int64_t gsize, int n_top, int32_t *idx) {
    __shared__ unsigned long long sel[kSelMaxTop];
    __shared__ uint32_t hist[256];
    __shared__ int s_warp[33];
    __shared__ uint32_t s_prefix, s_rank;
    __shared__ int s_cnt;
    const int tid = threadIdx.x;
    const float *v = vals ? vals + (int64_t)blockIdx.x * gsize * stride : nullptr;
    const TrialRes *rv = vals ? nullptr : res + (int64_t)blockIdx.x * gsize;
    if (tid == 0) {
        s_prefix = 0;
        s_rank = (uint32_t)n_top;
        s_cnt = 0;
    }
    // ---- radix select of the n_top-th largest key, 8 bits at a time from the top
    uint32_t mask = 0;
    for (int shift = 24; shift >= 0; shift -= 8) {
        for (int i = tid; i < 256; i += kSelThreads) hist[i] = 0;
        __syncthreads();
        const uint32_t prefix = s_prefix;
        for (int64_t i = tid; i < gsize; i += kSelThreads) {
            const uint32_t k = val_key(v, rv, stride, i);
            if ((k & mask) == prefix) atomicAdd(&hist[(k >> shift) & 255u], 1u);
        }
        __syncthreads();
        if (tid == 0) {
            uint32_t cum = 0, r = s_rank;
            for (int d = 255; d >= 0; --d) {
                if (cum + hist[d] >= r) {
                    s_rank = r - cum;  // rank within bucket d
                    s_prefix = prefix | ((uint32_t)d << shift);
                    break;
                }
                cum += hist[d];
            }
        }
        mask |= 255u << shift;
        __syncthreads();
    }
    // ---- rows above the threshold key, and the first s_rank rows equal to it (index order)
    const uint32_t thr = s_prefix;
    const int take_eq = (int)s_rank;
    int eq_seen = 0;
    for (int64_t base = 0; base < gsize; base += kSelThreads) {
        const int64_t i = base + tid;
        const uint32_t k = i < gsize ? val_key(v, rv, stride, i) : 0u;
        const bool gt = i < gsize && k > thr, eq = i < gsize && k == thr;
        int n_eq = 0;
        const int pre = block_prefix(eq, s_warp, &n_eq);
        const bool keep = gt || (eq && eq_seen + pre < take_eq);
        if (keep) {
            const int p = atomicAdd(&s_cnt, 1);
            sel[p] = ((unsigned long long)k << 32) | (0xffffffffu - (uint32_t)i);
        }
        eq_seen += n_eq;
    }
    __syncthreads();
    // ---- bitonic sort of the selected rows, descending by (key, -index)
    int n2 = 1;
    while (n2 < n_top) n2 <<= 1;
    for (int i = n_top + tid; i < n2; i += kSelThreads) sel[i] = 0ull;
    __syncthreads();
    for (int k = 2; k <= n2; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = tid; i < n2; i += kSelThreads) {
                const int l = i ^ j;
                if (l > i) {
                    const unsigned long long a = sel[i], b = sel[l];
                    const bool desc = (i & k) == 0;
                    if (desc ? a < b : a > b) {
                        sel[i] = b;
                        sel[l] = a;
                    }
                }
            }
            __syncthreads();
        }
    }
    for (int r = tid; r < n_top; r += kSelThreads)
        idx[(int64_t)blockIdx.x * n_top + r] = (int32_t)(0xffffffffu - (uint32_t)sel[r]);
}

// rows_out[g*n_top + k] (row_len values) = rows_src of the group's rank-k row (float32 rows widened
// to double, or double rows copied), when both are given.
__global__ void gather_rows_k(const int32_t *idx, int64_t n_groups, int n_top, int64_t gsize, const float *src_f,
                              const double *src_d, int64_t src_group_stride, int row_len, double *out) {
    const int64_t n = n_groups * n_top * row_len;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = e / row_len, c = e - r * row_len, g = r / n_top;
        const int64_t row = (int64_t)idx[r] + g * src_group_stride;
        out[e] = src_f ? (double)src_f[row * row_len + c] : src_d[row * row_len + c];
    }
}

__global__ void gather_floats_k(const int32_t *idx, int64_t n_groups, int n_top, const float *src, int64_t src_stride,
                                float *out) {
    const int64_t n = n_groups * n_top;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x)
        out[r] = src[(r / n_top) * src_stride + idx[r]];
}

// x0 of the first n_x0 sorted rows of every seed: (b, c, d) of [q0 b c d].
__global__ void take_x0_k(const double *rows, int64_t n, int k, int n_x0, double *x0) {
    const int64_t m = n * n_x0 * 3;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = e / 3, c = e - r * 3, sd = r / n_x0, j = r - sd * n_x0;
        x0[e] = rows[(sd * k + j) * 4 + 1 + c];
    }
}

// Lexicographic "a before b" of two grid rows (NaN after every number, as a stable numeric sort).
__device__ __forceinline__ bool row_before(const double *a, int ia, const double *b, int ib) {
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const double x = a[c], y = b[c];
        const bool nx = isnan(x), ny = isnan(y);
        if (nx != ny) return ny;  // the number goes first
        if (!nx && x != y) return x < y;
    }
    return ia < ib;
}

// One block per candidate: L = (nr+1)^3 + 1 rows (L <= kSelThreads), sorted in shared memory.
__global__ void __launch_bounds__(kSelThreads) local_grid_k(const double *cand, int64_t n_cand, int nr,
                                                            double gridsize, double half, double *out,
                                                            double *out_r32, float *out_f32) {
    __shared__ double rows[kSelThreads][4];
    __shared__ int ord[kSelThreads];
    const int tid = threadIdx.x, m = nr + 1, L = m * m * m + 1;
    const double *q = cand + 4 * (int64_t)blockIdx.x;
    int n2 = 1;
    while (n2 < L) n2 <<= 1;
    if (tid < L) {
        if (tid == 0) {
            for (int c = 0; c < 4; ++c) rows[0][c] = q[c];
        } else {
            const int j = tid - 1, ib = j / (m * m), ic = (j / m) % m, id = j % m;
            // steps = k * gridsize - gridsize * nr / 2; b = q1 + steps(ib), ...
            const double b = __dadd_rn(q[1], __dsub_rn(__dmul_rn((double)ib, gridsize), half));
            const double c = __dadd_rn(q[2], __dsub_rn(__dmul_rn((double)ic, gridsize), half));
            const double d = __dadd_rn(q[3], __dsub_rn(__dmul_rn((double)id, gridsize), half));
            const double s = __dadd_rn(__dadd_rn(__dmul_rn(b, b), __dmul_rn(c, c)), __dmul_rn(d, d));
            rows[tid][0] = __dsqrt_rn(__dsub_rn(1.0, s));
            rows[tid][1] = b;
            rows[tid][2] = c;
            rows[tid][3] = d;
        }
    }
    if (tid < n2) ord[tid] = tid < L ? tid : -1;  // -1: padding, sorts last
    __syncthreads();
    for (int k = 2; k <= n2; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            const int i = tid, l = i ^ j;
            if (i < n2 && l > i) {
                const int a = ord[i], b = ord[l];
                bool a_first;
                if (a < 0 || b < 0)
                    a_first = b < 0;
                else
                    a_first = row_before(rows[a], a, rows[b], b);
                const bool up = (i & k) == 0;  // ascending run
                if (up ? !a_first : a_first) {
                    ord[i] = b;
                    ord[l] = a;
                }
            }
            __syncthreads();
        }
    }
    if (tid < L) {
        const int r = ord[tid];
        double *o = out + ((int64_t)blockIdx.x * L + tid) * 4;
        for (int c = 0; c < 4; ++c) {
            o[c] = rows[r][c];
            // the row as the MEX receives it: rounded to float32
            const int64_t e = ((int64_t)blockIdx.x * L + tid) * 4 + c;
            if (out_r32) out_r32[e] = (double)(float)rows[r][c];
            if (out_f32) out_f32[e] = (float)rows[r][c];
        }
    }
}

// Trial lists of consecutive blocks: voxel[t] = t / per_voxel, orient[t] = t.
__global__ void block_lists_k(int64_t n, int64_t per_voxel, int32_t *voxel, int32_t *orient) {
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        voxel[t] = (int32_t)(t / per_voxel);
        orient[t] = (int32_t)t;
    }
}

}  // namespace

cudaError_t launch_block_lists(int64_t n, int64_t per_voxel, int32_t *voxel, int32_t *orient, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    const int64_t want = (n + 255) / 256;
    block_lists_k<<<(int)(want < 65535 * 8 ? want : 65535 * 8), 256, 0, s>>>(n, per_voxel, voxel, orient);
    return cudaGetLastError();
}

cudaError_t launch_top_rows(const float *vals, const TrialRes *res, int64_t stride, int64_t n_groups, int64_t gsize,
                            int n_top, int32_t *idx, cudaStream_t s) {
    if (n_groups <= 0 || n_top <= 0) return cudaSuccess;
    if (n_top > kSelMaxTop || n_top > gsize || n_groups > 2147483647LL || (!vals && !res))
        return cudaErrorInvalidValue;
    top_rows_k<<<(unsigned)n_groups, kSelThreads, 0, s>>>(vals, res, stride, gsize, n_top, idx);
    return cudaGetLastError();
}

cudaError_t launch_gather_rows(const int32_t *idx, int64_t n_groups, int n_top, int64_t gsize, const float *src_f,
                               const double *src_d, int64_t src_group_stride, int row_len, double *out,
                               cudaStream_t s) {
    const int64_t n = n_groups * n_top * row_len;
    if (n <= 0) return cudaSuccess;
    const int64_t want = (n + 255) / 256;
    gather_rows_k<<<(int)(want < 65535 * 8 ? want : 65535 * 8), 256, 0, s>>>(idx, n_groups, n_top, gsize, src_f,
                                                                          src_d, src_group_stride, row_len, out);
    return cudaGetLastError();
}

cudaError_t launch_gather_floats(const int32_t *idx, int64_t n_groups, int n_top, int64_t gsize, const float *src,
                                 int64_t src_stride, float *out, cudaStream_t s) {
    const int64_t n = n_groups * n_top;
    if (n <= 0) return cudaSuccess;
    const int64_t want = (n + 255) / 256;
    gather_floats_k<<<(int)(want < 65535 * 8 ? want : 65535 * 8), 256, 0, s>>>(idx, n_groups, n_top, src, src_stride,
                                                                            out);
    return cudaGetLastError();
}

cudaError_t launch_take_x0(const double *rows, int64_t n, int k, int n_x0, double *x0, cudaStream_t s) {
    const int64_t m = n * n_x0 * 3;
    if (m <= 0) return cudaSuccess;
    const int64_t want = (m + 255) / 256;
    take_x0_k<<<(int)(want < 65535 * 8 ? want : 65535 * 8), 256, 0, s>>>(rows, n, k, n_x0, x0);
    return cudaGetLastError();
}

int local_grid_rows(int nr) { return (nr + 1) * (nr + 1) * (nr + 1) + 1; }

cudaError_t launch_local_grid(const double *cand, int64_t n_cand, int nr, double gridsize, double *out,
                              double *out_r32, float *out_f32, cudaStream_t s) {
    if (n_cand <= 0) return cudaSuccess;
    if (nr < 0 || local_grid_rows(nr) > kSelThreads || n_cand > 2147483647LL) return cudaErrorInvalidValue;
    const double half = gridsize * nr / 2;
    local_grid_k<<<(unsigned)n_cand, kSelThreads, 0, s>>>(cand, n_cand, nr, gridsize, half, out, out_r32, out_f32);
    return cudaGetLastError();
}

}  // namespace grc
