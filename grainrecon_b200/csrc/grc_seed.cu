// grc_seed.cu -- trial lists in FP64 and the batched orientation fit of the seeding stage.
//
// The seeding engine (GrainMapping_engine_gpu_comp.m:54-331) refines each seed's best
// orientation by a bounded Nelder-Mead on 1 - completeness (fminsearchbnd over q1..q3,
// fit_OR_constrain_with_local_comp_cuda.m:115-157, objective fit_OR_fun_local.m:2-98).
// Here every seed of a batch runs its own simplex; one step proposes up to four points per
// seed, the scorer evaluates all of them in one launch, and a second kernel applies the
// fminsearch rules.  Reflection, expansion and both contractions are scored together and
// only the points the sequential algorithm would have evaluated are counted, so each
// simplex follows the sequential trajectory exactly.
#include <cuda_runtime.h>
#include <float.h>
#include <math_constants.h>
#include <stdint.h>

#include "grc_internal.h"

namespace grc {
namespace {

constexpr int kB = 256;

inline int blocks_for(int64_t n) {
    int64_t b = (n + kB - 1) / kB;
    if (b < 1) b = 1;
    if (b > (1 << 30)) b = 1 << 30;
    return (int)b;
}

// Rounded double arithmetic without contraction, so host and device agree bit for bit.
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }

// fit_OR_fun_local.m:8-25 (= quaternion2U.m): q0 = sqrt(1 - (q1^2 + q2^2 + q3^2)), U from q.
__device__ void quat_u(double q0, double q1, double q2, double q3, double *u) {
    u[0] = sub(mul(2.0, add(mul(q0, q0), mul(q1, q1))), 1.0);
    u[1] = mul(2.0, sub(mul(q1, q2), mul(q0, q3)));
    u[2] = mul(2.0, add(mul(q1, q3), mul(q0, q2)));
    u[3] = mul(2.0, add(mul(q1, q2), mul(q0, q3)));
    u[4] = sub(mul(2.0, add(mul(q0, q0), mul(q2, q2))), 1.0);
    u[5] = mul(2.0, sub(mul(q2, q3), mul(q0, q1)));
    u[6] = mul(2.0, sub(mul(q1, q3), mul(q0, q2)));
    u[7] = mul(2.0, add(mul(q2, q3), mul(q0, q1)));
    u[8] = sub(mul(2.0, add(mul(q0, q0), mul(q3, q3))), 1.0);
}

__global__ void quat_to_u_d_k(const double *q, int64_t n, double *U) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        quat_u(q[4 * i], q[4 * i + 1], q[4 * i + 2], q[4 * i + 3], U + 9 * i);
}

__global__ void trial_items_k(const int32_t *tv, const int32_t *to, int64_t n, int64_t n_vox, int64_t n_q,
                              longlong4 *items, int *bad) {
    // blockDim is a multiple of 32, so each warp walks aligned blocks of 32 trials; the loop test
    // uses the block's first trial, so all lanes of a warp take part in every ballot
    const int lane = threadIdx.x & 31;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i - lane < n; i += (int64_t)gridDim.x * blockDim.x) {
        const bool in = i < n;
        bool start = false;
        if (in) {
            const int64_t v = tv[i], o = to[i];
            const bool ok = v >= 0 && v < n_vox && o >= 0 && o < n_q;
            if (!ok) atomicOr(bad, 1);
            items[i] = make_longlong4(ok ? v : 0, i, ok ? i + 1 : i, 0);
            start = i == 0 || tv[i] != tv[i - 1];
        }
        const int starts = __popc(__ballot_sync(0xffffffffu, start));
        if (lane == 0 && starts > 0) atomicMax(bad + 1, starts);
    }
}

// ---- spot index and pair ordering ----------------------------------------------------------

// One block per projection: cell key and count of every spot (centroids outside the detector
// fall into the border cells).
__global__ void spot_keys_k(const double *yza, const int64_t *proj_off, int ncy, int ncz, int cell_px,
                            int32_t *keys, int32_t *ids, int64_t *cell_counts) {
    const int iw = blockIdx.x;
    for (int64_t i = proj_off[iw] + threadIdx.x; i < proj_off[iw + 1]; i += blockDim.x) {
        const double cy = floor((yza[3 * i] - 1.0) / cell_px), cz = floor((yza[3 * i + 1] - 1.0) / cell_px);
        const int y = cy < 0.0 ? 0 : (cy > ncy - 1 ? ncy - 1 : (int)cy);
        const int z = cz < 0.0 ? 0 : (cz > ncz - 1 ? ncz - 1 : (int)cz);
        const int32_t key = (iw * ncy + y) * ncz + z;
        keys[i] = key;
        ids[i] = (int32_t)i;
        atomicAdd((unsigned long long *)(cell_counts + key), 1ull);
    }
}

__global__ void pair_keys_k(const PairRec *p, int64_t n, int nrot, int nhkl, int64_t *keys, int32_t *ids) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        keys[i] = ((int64_t)p[i].trial * nrot + p[i].iw) * nhkl + p[i].ih;
        ids[i] = (int32_t)i;
    }
}

__global__ void pair_gather_k(const PairRec *in, const int32_t *order, int64_t n, PairRec *out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = in[order[i]];
}

// ---- batched fminsearchbnd -------------------------------------------------------------

enum : int { kInit = 0, kNormal = 1, kShrink = 2, kDone = 3 };

__device__ __forceinline__ bool before(double a, double b) {  // ascending, NaN last (MATLAB sort)
    return a < b || (!isnan(a) && isnan(b));
}

__device__ __forceinline__ double nanmax2(double a, double b) {  // MATLAB max ignores NaN
    if (isnan(a)) return b;
    if (isnan(b)) return a;
    return a > b ? a : b;
}

// MATLAB eps(x): distance from |x| to the next larger double.
__device__ double eps_of(double x) {
    x = fabs(x);
    if (!(x <= DBL_MAX)) return CUDART_NAN;
    if (x < DBL_MIN) return 4.9406564584124654e-324;
    int e;
    frexp(x, &e);  // x = m * 2^e, m in [0.5, 1)
    return ldexp(1.0, e - 53);
}

// fminsearchbnd.m:245-268, both bounds given: x = LB + (UB - LB) (sin z + 1) / 2, clamped.
__device__ void xtransform(const NmSeed &s, const double *z, double *x) {
    for (int k = 0; k < 3; ++k) {
        double t = mul(add(sin(z[k]), 1.0), 0.5);
        t = add(mul(t, sub(s.ub[k], s.lb[k])), s.lb[k]);
        x[k] = fmax(s.lb[k], fmin(s.ub[k], t));
    }
}

__device__ void sort4(NmSeed &s) {
    for (int i = 1; i < 4; ++i) {
        const double f = s.fv[i];
        double z[3] = {s.z[i][0], s.z[i][1], s.z[i][2]};
        int j = i - 1;
        while (j >= 0 && before(f, s.fv[j])) {
            s.fv[j + 1] = s.fv[j];
            for (int k = 0; k < 3; ++k) s.z[j + 1][k] = s.z[j][k];
            --j;
        }
        s.fv[j + 1] = f;
        for (int k = 0; k < 3; ++k) s.z[j + 1][k] = z[k];
    }
}

// 1 - Nr_intersect / Nr_simu in FP64 (fit_OR_fun_local.m:97); NaN when nothing is simulated
// or when the slot's point had no real q0 (bit j of nanmask).
__device__ __forceinline__ double objective(const NmSeed &s, const TrialRes *r, int j) {
    if (s.nanmask & (1 << j)) return CUDART_NAN;
    return sub(1.0, (double)r[j].inter / (double)r[j].simu);
}

__global__ void nm_init_k(NmSeed *st, int64_t n, const double *x0, double half_width) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        NmSeed s;
        double z0[3];
        for (int k = 0; k < 3; ++k) {
            const double x = x0[3 * i + k];
            // fit_OR_constrain_with_local_comp_cuda.m:124-125
            s.lb[k] = fmax(sub(x, half_width), -1.0);
            s.ub[k] = fmin(add(x, half_width), 1.0);
            // fminsearchbnd.m:152-165: interior start -> 2*pi + asin(2 (x - LB)/(UB - LB) - 1)
            if (x <= s.lb[k]) {
                z0[k] = -CUDART_PIO2;
            } else if (x >= s.ub[k]) {
                z0[k] = CUDART_PIO2;
            } else {
                const double u = sub(mul(2.0, sub(x, s.lb[k])) / sub(s.ub[k], s.lb[k]), 1.0);
                z0[k] = add(2.0 * CUDART_PI, asin(fmax(-1.0, fmin(1.0, u))));
            }
        }
        // fminsearch initial simplex: x0 and x0 with one coordinate scaled by 1.05
        // (0.00025 when that coordinate is zero)
        for (int v = 0; v < 4; ++v)
            for (int k = 0; k < 3; ++k) s.cand[v][k] = z0[k];
        for (int k = 0; k < 3; ++k)
            s.cand[k + 1][k] = z0[k] != 0.0 ? mul(add(1.0, 0.05), z0[k]) : 0.00025;
        for (int v = 0; v < 4; ++v) s.fv[v] = CUDART_NAN;
        s.evals = 0;
        s.iters = 0;
        s.phase = kInit;
        s.flag = 0;
        s.nanmask = 0;
        st[i] = s;
    }
}

// One step, first half: decide termination and write the points to evaluate as U matrices
// (trial 4i + j of seed i) and work items (empty items for unused slots).
__global__ void nm_propose_k(NmSeed *st, int64_t n, int max_evals, int max_iter, double tol_f, double tol_x,
                             double *U, longlong4 *items, int *active) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        NmSeed &s = st[i];
        int n_eval = 0;
        if (s.phase == kNormal) {
            // fminsearch loop head: limits, then the TolFun / TolX test on the sorted simplex
            if (s.evals >= max_evals || s.iters >= max_iter) {
                s.phase = kDone;
                s.flag = 0;
            } else {
                double df = CUDART_NAN, dx = CUDART_NAN, zmax = CUDART_NAN;
                for (int v = 1; v < 4; ++v) {
                    df = nanmax2(df, fabs(sub(s.fv[0], s.fv[v])));
                    for (int k = 0; k < 3; ++k) dx = nanmax2(dx, fabs(sub(s.z[v][k], s.z[0][k])));
                }
                for (int k = 0; k < 3; ++k) zmax = nanmax2(zmax, s.z[0][k]);
                const double tf = nanmax2(tol_f, mul(10.0, eps_of(s.fv[0])));
                const double tx = nanmax2(tol_x, mul(10.0, eps_of(zmax)));
                if (df <= tf && dx <= tx) {
                    s.phase = kDone;
                    s.flag = 1;
                }
            }
            if (s.phase == kNormal) {
                // centroid of the best three, then reflection / expansion / contractions
                double xb[3];
                for (int k = 0; k < 3; ++k) xb[k] = add(add(s.z[0][k], s.z[1][k]), s.z[2][k]) / 3.0;
                for (int k = 0; k < 3; ++k) {
                    const double w = s.z[3][k];
                    s.cand[0][k] = sub(mul(2.0, xb[k]), mul(1.0, w));     // (1+rho) xbar - rho w
                    s.cand[1][k] = sub(mul(3.0, xb[k]), mul(2.0, w));     // (1+rho chi) xbar - rho chi w
                    s.cand[2][k] = sub(mul(1.5, xb[k]), mul(0.5, w));     // (1+psi rho) xbar - psi rho w
                    s.cand[3][k] = add(mul(0.5, xb[k]), mul(0.5, w));     // (1-psi) xbar + psi w
                }
                n_eval = 4;
            }
        } else if (s.phase == kInit) {
            n_eval = 4;
        } else if (s.phase == kShrink) {
            for (int v = 0; v < 3; ++v)
                for (int k = 0; k < 3; ++k) s.cand[v][k] = s.z[v + 1][k];
            n_eval = 3;
        }
        if (s.phase != kDone) atomicAdd(active, 1);
        s.nanmask = 0;
        for (int j = 0; j < 4; ++j) {
            const int64_t t = 4 * i + j;
            bool on = j < n_eval;
            if (on) {
                double x[3];
                xtransform(s, s.cand[j], x);
                const double r2 = add(add(mul(x[0], x[0]), mul(x[1], x[1])), mul(x[2], x[2]));
                if (r2 <= 1.0) {
                    quat_u(sqrt(sub(1.0, r2)), x[0], x[1], x[2], U + 9 * t);
                } else {  // q0 would be imaginary: the objective is NaN, nothing is scored
                    s.nanmask |= 1 << j;
                    on = false;
                }
            }
            items[t] = make_longlong4(i, t, on ? t + 1 : t, 0);
        }
    }
}

// One step, second half: the fminsearch update with the scored points.
__global__ void nm_accept_k(NmSeed *st, int64_t n, const TrialRes *res) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        NmSeed &s = st[i];
        const TrialRes *r = res + 4 * i;
        if (s.phase == kInit) {
            for (int v = 0; v < 4; ++v) {
                s.fv[v] = objective(s, r, v);
                for (int k = 0; k < 3; ++k) s.z[v][k] = s.cand[v][k];
            }
            sort4(s);
            s.evals = 4;
            s.iters = 1;
            s.phase = kNormal;
        } else if (s.phase == kShrink) {
            for (int v = 1; v < 4; ++v) s.fv[v] = objective(s, r, v - 1);
            s.evals += 3;
            sort4(s);
            s.iters += 1;
            s.phase = kNormal;
        } else if (s.phase == kNormal) {
            const double fr = objective(s, r, 0);
            s.evals += 1;
            int take = -1;  // candidate replacing the worst vertex; -2 = shrink
            if (fr < s.fv[0]) {
                const double fe = objective(s, r, 1);
                s.evals += 1;
                take = fe < fr ? 1 : 0;
            } else if (fr < s.fv[2]) {
                take = 0;
            } else if (fr < s.fv[3]) {
                const double fc = objective(s, r, 2);
                s.evals += 1;
                take = fc <= fr ? 2 : -2;
            } else {
                const double fcc = objective(s, r, 3);
                s.evals += 1;
                take = fcc < s.fv[3] ? 3 : -2;
            }
            if (take >= 0) {
                for (int k = 0; k < 3; ++k) s.z[3][k] = s.cand[take][k];
                s.fv[3] = objective(s, r, take);
                sort4(s);
                s.iters += 1;
            } else {
                for (int v = 1; v < 4; ++v)
                    for (int k = 0; k < 3; ++k)
                        s.z[v][k] = add(s.z[0][k], mul(0.5, sub(s.z[v][k], s.z[0][k])));
                s.phase = kShrink;
            }
        }
    }
}

__global__ void nm_final_k(const NmSeed *st, int64_t n, double *x, double *fval, int32_t *evals, int32_t *iters,
                           int32_t *flag) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const NmSeed &s = st[i];
        double xo[3];
        xtransform(s, s.z[0], xo);
        for (int k = 0; k < 3; ++k) x[3 * i + k] = xo[k];
        fval[i] = s.fv[0];
        if (evals) evals[i] = s.evals;
        if (iters) iters[i] = s.iters;
        if (flag) flag[i] = s.phase == kDone ? s.flag : -1;
    }
}

}  // namespace

cudaError_t launch_quat_to_u_d(const double *q, int64_t n, double *U, cudaStream_t s) {
    quat_to_u_d_k<<<blocks_for(n), kB, 0, s>>>(q, n, U);
    return cudaGetLastError();
}

cudaError_t launch_trial_items(const int32_t *tv, const int32_t *to, int64_t n, int64_t n_vox, int64_t n_q,
                               longlong4 *items, int *bad, cudaStream_t s) {
    trial_items_k<<<blocks_for(n), kB, 0, s>>>(tv, to, n, n_vox, n_q, items, bad);
    return cudaGetLastError();
}

cudaError_t launch_spot_keys(const double *yza, const int64_t *proj_off, int nrot, int ncy, int ncz, int cell_px,
                             int32_t *keys, int32_t *ids, int64_t *cell_counts, cudaStream_t s) {
    spot_keys_k<<<nrot, kB, 0, s>>>(yza, proj_off, ncy, ncz, cell_px, keys, ids, cell_counts);
    return cudaGetLastError();
}

cudaError_t launch_pair_keys(const PairRec *p, int64_t n, int nrot, int nhkl, int64_t *keys, int32_t *ids,
                             cudaStream_t s) {
    pair_keys_k<<<blocks_for(n), kB, 0, s>>>(p, n, nrot, nhkl, keys, ids);
    return cudaGetLastError();
}

cudaError_t launch_pair_gather(const PairRec *in, const int32_t *order, int64_t n, PairRec *out, cudaStream_t s) {
    pair_gather_k<<<blocks_for(n), kB, 0, s>>>(in, order, n, out);
    return cudaGetLastError();
}

cudaError_t launch_nm_init(NmSeed *st, int64_t n, const double *x0, double half_width, cudaStream_t s) {
    nm_init_k<<<blocks_for(n), kB, 0, s>>>(st, n, x0, half_width);
    return cudaGetLastError();
}

cudaError_t launch_nm_propose(NmSeed *st, int64_t n, int max_evals, int max_iter, double tol_f, double tol_x,
                              double *U, longlong4 *items, int *active, cudaStream_t s) {
    nm_propose_k<<<blocks_for(n), kB, 0, s>>>(st, n, max_evals, max_iter, tol_f, tol_x, U, items, active);
    return cudaGetLastError();
}

cudaError_t launch_nm_accept(NmSeed *st, int64_t n, const TrialRes *res, cudaStream_t s) {
    nm_accept_k<<<blocks_for(n), kB, 0, s>>>(st, n, res);
    return cudaGetLastError();
}

namespace {
__global__ void nm_continue_k(cudaGraphConditionalHandle handle, const int *active, int *bodies, int max_bodies) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        const int k = ++*bodies;
        cudaGraphSetConditional(handle, (*active > 0 && k < max_bodies) ? 1u : 0u);
    }
}
}  // namespace

cudaError_t launch_nm_continue(unsigned long long handle, const int *active, int *bodies, int max_bodies,
                               cudaStream_t s) {
    nm_continue_k<<<1, 32, 0, s>>>((cudaGraphConditionalHandle)handle, active, bodies, max_bodies);
    return cudaGetLastError();
}

cudaError_t launch_nm_final(const NmSeed *st, int64_t n, double *x, double *fval, int32_t *evals, int32_t *iters,
                            int32_t *flag, cudaStream_t s) {
    nm_final_k<<<blocks_for(n), kB, 0, s>>>(st, n, x, fval, evals, iters, flag);
    return cudaGetLastError();
}

}  // namespace grc
