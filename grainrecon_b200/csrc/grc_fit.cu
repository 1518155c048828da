// grc_fit.cu -- derivatives of the continuous spot-centroid residual and the fits they drive.
//
// The reference fits grain orientation/centre (fit_grain_COM.m:5-88,
// fit_OR_fun_local.m) and the detector geometry (geo_fitting.m:5-78,
// L_shift_tilt_fitting.m:23-50) with fminsearchbnd (Nelder-Mead) on discrete
// objectives (rounded pixels, 1-completeness).  Here the residual is the continuous
// landing point (u, v) of forward_comp.m:28-59 -- no rounding -- minus the measured
// spot centroid, for a fixed set of matched (grain, omega, hkl) spots.
//
// Derivatives are hand-propagated tangents: the landing chain is written once over a
// dual-number scalar (value + KC tangent components) and evaluated in FP64; the
// Jacobian of (u, v) with respect to the grain parameters (Rodrigues vector, centre)
// or the 10 geometry parameters (Lsam2sou, Lsam2det, dety00, detz00, tilt_x/y/z,
// P0y, P0z, RotAxisOffset) is assembled from ceil(K/KC) passes.  The gradient of the
// least-squares loss is J^T r.  Normal equations are accumulated in FP64 and solved
// per grain (6x6) or per start (10x10) with Levenberg-Marquardt damping.
#include <cuda_runtime.h>
#include <math_constants.h>
#include <stdint.h>

#include "grc_fit.h"
#include "grc_internal.h"

namespace grc {
namespace {

// ---- dual numbers ----------------------------------------------------------------
template <int K>
struct D {
    double v;
    double d[K > 0 ? K : 1];
};

template <int K>
__host__ __device__ __forceinline__ D<K> cst(double x) {
    D<K> r;
    r.v = x;
#pragma unroll
    for (int i = 0; i < K; ++i) r.d[i] = 0.0;
    return r;
}
template <int K>
__host__ __device__ __forceinline__ D<K> operator+(const D<K> &a, const D<K> &b) {
    D<K> r;
    r.v = a.v + b.v;
#pragma unroll
    for (int i = 0; i < K; ++i) r.d[i] = a.d[i] + b.d[i];
    return r;
}
template <int K>
__host__ __device__ __forceinline__ D<K> operator-(const D<K> &a, const D<K> &b) {
    D<K> r;
    r.v = a.v - b.v;
#pragma unroll
    for (int i = 0; i < K; ++i) r.d[i] = a.d[i] - b.d[i];
    return r;
}
template <int K>
__host__ __device__ __forceinline__ D<K> operator-(const D<K> &a) {
    D<K> r;
    r.v = -a.v;
#pragma unroll
    for (int i = 0; i < K; ++i) r.d[i] = -a.d[i];
    return r;
}
template <int K>
__host__ __device__ __forceinline__ D<K> operator*(const D<K> &a, const D<K> &b) {
    D<K> r;
    r.v = a.v * b.v;
#pragma unroll
    for (int i = 0; i < K; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
    return r;
}
template <int K>
__host__ __device__ __forceinline__ D<K> operator*(const D<K> &a, double b) {
    D<K> r;
    r.v = a.v * b;
#pragma unroll
    for (int i = 0; i < K; ++i) r.d[i] = a.d[i] * b;
    return r;
}
template <int K>
__host__ __device__ __forceinline__ D<K> operator*(double b, const D<K> &a) {
    return a * b;
}
template <int K>
__host__ __device__ __forceinline__ D<K> operator+(const D<K> &a, double b) {
    D<K> r = a;
    r.v += b;
    return r;
}
template <int K>
__host__ __device__ __forceinline__ D<K> operator+(double b, const D<K> &a) {
    return a + b;
}
template <int K>
__host__ __device__ __forceinline__ D<K> operator-(const D<K> &a, double b) {
    D<K> r = a;
    r.v -= b;
    return r;
}
template <int K>
__host__ __device__ __forceinline__ D<K> operator-(double b, const D<K> &a) {
    return -a + b;
}
template <int K>
__host__ __device__ __forceinline__ D<K> operator/(const D<K> &a, const D<K> &b) {
    D<K> r;
    const double ib = 1.0 / b.v;
    r.v = a.v * ib;
#pragma unroll
    for (int i = 0; i < K; ++i) r.d[i] = (a.d[i] - r.v * b.d[i]) * ib;
    return r;
}
template <int K>
__host__ __device__ __forceinline__ D<K> operator/(const D<K> &a, double b) {
    return a * (1.0 / b);
}
template <int K>
__host__ __device__ __forceinline__ D<K> operator/(double a, const D<K> &b) {
    return cst<K>(a) / b;
}
template <int K>
__host__ __device__ __forceinline__ D<K> dsqrt(const D<K> &a) {
    D<K> r;
    r.v = sqrt(a.v);
    const double h = 0.5 / r.v;
#pragma unroll
    for (int i = 0; i < K; ++i) r.d[i] = a.d[i] * h;
    return r;
}
template <int K>
__host__ __device__ __forceinline__ D<K> dsin(const D<K> &a) {
    D<K> r;
    r.v = sin(a.v);
    const double c = cos(a.v);
#pragma unroll
    for (int i = 0; i < K; ++i) r.d[i] = a.d[i] * c;
    return r;
}
template <int K>
__host__ __device__ __forceinline__ D<K> dcos(const D<K> &a) {
    D<K> r;
    r.v = cos(a.v);
    const double s = -sin(a.v);
#pragma unroll
    for (int i = 0; i < K; ++i) r.d[i] = a.d[i] * s;
    return r;
}

// ---- the landing chain --------------------------------------------------------------
// Grain parameters g[0..2] = Rodrigues vector r (U from q0 = 1/sqrt(1+|r|^2), q = r q0 via
// quaternion2U.m:3-28), g[3..5] = centre [mm].  Geometry e[0..9] = Lsam2sou, Lsam2det,
// dety00, detz00, tilt_x, tilt_y, tilt_z [deg], P0y, P0z, RotAxisOffset; RotDet =
// Rz*Ry*Rx (get_det_R.m:1-7).  (u, v) are the unrounded pixel coordinates of
// forward_comp.m:58-59.  strict: false when the reflection is outside the wavelength /
// Bragg-angle window or the detector (decides which spots exist); otherwise false only
// for a non-finite landing (a matched spot stays in the residual during a fit).
template <int K>
__device__ __forceinline__ bool uv_chain(const FitFixed &fx, const D<K> *g, const D<K> *e, double c, double s,
                                         const double *h, D<K> &u, D<K> &v, bool strict) {
    // U
    const D<K> rr = g[0] * g[0] + g[1] * g[1] + g[2] * g[2];
    const D<K> q0 = 1.0 / dsqrt(1.0 + rr);
    const D<K> q1 = g[0] * q0, q2 = g[1] * q0, q3 = g[2] * q0;
    D<K> U[9];
    U[0] = 2.0 * (q0 * q0 + q1 * q1) - 1.0;
    U[1] = 2.0 * (q1 * q2 - q0 * q3);
    U[2] = 2.0 * (q1 * q3 + q0 * q2);
    U[3] = 2.0 * (q1 * q2 + q0 * q3);
    U[4] = 2.0 * (q0 * q0 + q2 * q2) - 1.0;
    U[5] = 2.0 * (q2 * q3 - q0 * q1);
    U[6] = 2.0 * (q1 * q3 - q0 * q2);
    U[7] = 2.0 * (q2 * q3 + q0 * q1);
    U[8] = 2.0 * (q0 * q0 + q3 * q3) - 1.0;
    // Gw = S U B h
    const double bh0 = fx.B[0] * h[0] + fx.B[1] * h[1] + fx.B[2] * h[2];
    const double bh1 = fx.B[3] * h[0] + fx.B[4] * h[1] + fx.B[5] * h[2];
    const double bh2 = fx.B[6] * h[0] + fx.B[7] * h[1] + fx.B[8] * h[2];
    const D<K> ub0 = U[0] * bh0 + U[1] * bh1 + U[2] * bh2;
    const D<K> ub1 = U[3] * bh0 + U[4] * bh1 + U[5] * bh2;
    const D<K> ub2 = U[6] * bh0 + U[7] * bh1 + U[8] * bh2;
    const D<K> gw0 = fx.S[0] * ub0 + fx.S[1] * ub1 + fx.S[2] * ub2;
    const D<K> gw1 = fx.S[3] * ub0 + fx.S[4] * ub1 + fx.S[5] * ub2;
    const D<K> gw2 = fx.S[6] * ub0 + fx.S[7] * ub1 + fx.S[8] * ub2;
    const D<K> Gtx = c * gw0 - s * gw1, Gty = s * gw0 + c * gw1, Gtz = gw2;
    const D<K> G = dsqrt(Gtx * Gtx + Gty * Gty + Gtz * Gtz);
    // sample point and incident beam (forward_comp.m:17-26)
    const D<K> &lss = e[0], &lsd = e[1], &y00 = e[2], &z00 = e[3], &p0y = e[7], &p0z = e[8], &rao = e[9];
    const D<K> px = g[3], py = g[4] - rao, pz = g[5];
    const D<K> spx = fx.S[0] * px + fx.S[1] * py + fx.S[2] * pz;
    const D<K> spy = fx.S[3] * px + fx.S[4] * py + fx.S[5] * pz;
    const D<K> spz = fx.S[6] * px + fx.S[7] * py + fx.S[8] * pz;
    const D<K> swx = c * spx - s * spy, swy = s * spx + c * spy, swz = spz;
    const D<K> gpx = lss + swx, gpy = swy - p0y + rao, gpz = swz - p0z;
    const D<K> ngp = dsqrt(gpx * gpx + gpy * gpy + gpz * gpz);
    const D<K> kx = gpx / ngp, ky = gpy / ngp, kz = gpz / ngp;
    const D<K> L = lss + lsd;
    const D<K> L2 = (lsd - swx) * ngp / gpx;
    const D<K> ax = lsd - swx, ay = gpy * L / gpx - swy, az = gpz * L / gpx - swz;
    // Bragg condition (forward_comp.m:28-37)
    const D<K> x = (kx * Gtx + ky * Gty + kz * Gtz) / G;
    const double lam = 2.0 * (2.0 * CUDART_PI / G.v) * (-x.v);
    if (strict && !(x.v < 0.0 && x.v > fx.cbmax && lam > fx.lmin && lam < fx.lmax)) return false;
    const D<K> st = -x, ct = dsqrt(1.0 - x * x);
    const D<K> s2 = 2.0 * st * ct, c2 = 1.0 - 2.0 * st * st;
    const D<K> konst = dsqrt(Gty * Gty + Gtz * Gtz);
    const D<K> gy = Gty / konst, gz = Gtz / konst;
    const D<K> cphx = gy * ky + gz * kz;
    const D<K> sphx = dsqrt(1.0 - cphx * cphx);
    const D<K> sphy = sphx * c2 - cphx * s2;
    const D<K> diff = L2 * s2 / sphy;
    const D<K> Kx = ax, Ky = ay + diff * gy, Kz = az + diff * gz;
    // tilted detector (forward_comp.m:49-55), RotDet from the tilts
    const double d2r = CUDART_PI / 180.0;
    const D<K> cxx = dcos(e[4] * d2r), sxx = dsin(e[4] * d2r);
    const D<K> cyy = dcos(e[5] * d2r), syy = dsin(e[5] * d2r);
    const D<K> czz = dcos(e[6] * d2r), szz = dsin(e[6] * d2r);
    // R = Rz*Ry*Rx, columns needed: R(:,1), R(:,2), R(:,3)
    const D<K> R00 = czz * cyy, R10 = szz * cyy, R20 = -syy;
    const D<K> R01 = czz * syy * sxx - szz * cxx, R11 = szz * syy * sxx + czz * cxx, R21 = cyy * sxx;
    const D<K> R02 = czz * syy * cxx + szz * sxx, R12 = szz * syy * cxx - czz * sxx, R22 = cyy * cxx;
    const D<K> dx = swx - lsd, dy = swy - y00 + rao, dz = swz - z00;
    const D<K> num = -(R00 * dx + R10 * dy + R20 * dz);
    const D<K> nK = R00 * Kx + R10 * Ky + R20 * Kz;
    const D<K> f = num / nK;
    const D<K> y2 = f * (R01 * Kx + R11 * Ky + R21 * Kz) + (R01 * dx + R11 * dy + R21 * dz);
    const D<K> z2 = f * (R02 * Kx + R12 * Ky + R22 * Kz) + (R02 * dx + R12 * dy + R22 * dz);
    u = fx.dety0 - y2 / fx.pxy;
    v = fx.detz0 - z2 / fx.pxz;
    if (!strict) return isfinite(u.v) && isfinite(v.v);
    return u.v >= 0.5 && u.v < fx.detysize + 0.5 && v.v >= 0.5 && v.v < fx.detzsize + 0.5;
}

// Residual and one KC-wide block of Jacobian columns [c0, c0+KC) of spot i.
// mode 0: columns over the 6 grain parameters; mode 1: over the 10 geometry parameters.
template <int KC>
__device__ __forceinline__ bool spot_eval(const FitFixed &fx, int mode, int c0, const double *grain6,
                                          const double *geo10, int iw, int ih, double &ru, double &rv,
                                          double *ju, double *jv, bool strict = false) {
    D<KC> g[6], e[10];
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        g[k] = cst<KC>(grain6[k]);
        if (mode == 0 && k >= c0 && k < c0 + KC) g[k].d[k - c0] = 1.0;
    }
#pragma unroll
    for (int k = 0; k < 10; ++k) {
        e[k] = cst<KC>(geo10[k]);
        if (mode == 1 && k >= c0 && k < c0 + KC) e[k].d[k - c0] = 1.0;
    }
    const double2 cs = fx.rot_cs[iw];
    const double h[3] = {fx.hkl[3 * ih], fx.hkl[3 * ih + 1], fx.hkl[3 * ih + 2]};
    D<KC> u, v;
    const bool ok = uv_chain<KC>(fx, g, e, cs.x, cs.y, h, u, v, strict);
    ru = u.v;
    rv = v.v;
#pragma unroll
    for (int k = 0; k < KC; ++k) {
        ju[k] = u.d[k];
        jv[k] = v.d[k];
    }
    return ok;
}

__device__ __forceinline__ bool spot_value(const FitFixed &fx, const double *grain6, const double *geo10, int iw,
                                           int ih, double &u, double &v, bool strict = false) {
    double ju[1], jv[1];
    return spot_eval<0>(fx, 0, 0, grain6, geo10, iw, ih, u, v, ju, jv, strict);
}

// ---- kernels -------------------------------------------------------------------------

// Per-spot residual (model - measured) and full Jacobian rows (2 x K).
template <int KC>
__global__ void residual_jac_k(FitFixed fx, int mode, const double *grains, const double *geo10, SpotList sp,
                               double *res, double *jac) {
    const int K = mode == 0 ? 6 : 10;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < sp.n; i += (int64_t)gridDim.x * blockDim.x) {
        const double *g6 = grains + 6 * (int64_t)sp.grain[i];
        double ru = 0, rv = 0, ju[KC], jv[KC];
        bool ok = true;
        for (int c0 = 0; c0 < K; c0 += KC) {
            ok = spot_eval<KC>(fx, mode, c0, g6, geo10, sp.iw[i], sp.ih[i], ru, rv, ju, jv);
            for (int k = 0; k < KC && c0 + k < K; ++k) {
                jac[(2 * i) * K + c0 + k] = ju[k];
                jac[(2 * i + 1) * K + c0 + k] = jv[k];
            }
        }
        res[2 * i] = ok ? ru - sp.uv[2 * i] : CUDART_NAN;
        res[2 * i + 1] = ok ? rv - sp.uv[2 * i + 1] : CUDART_NAN;
    }
}

// Block reduction of n doubles per thread into out (thread 0 holds the sums).
template <int N>
__device__ __forceinline__ void block_sum(double (&a)[N], double *scratch) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < N; ++k)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) a[k] += __shfl_down_sync(0xffffffffu, a[k], o);
    __syncthreads();
    if (lane == 0)
        for (int k = 0; k < N; ++k) scratch[warp * N + k] = a[k];
    __syncthreads();
    if (threadIdx.x == 0)
        for (int k = 0; k < N; ++k) {
            double t = 0;
            for (int w = 0; w < nw; ++w) t += scratch[w * N + k];
            a[k] = t;
        }
    __syncthreads();
}

// Normal equations of one grain per CTA: A = J^T J (21 upper), b = J^T r (6), c = r^T r, n.
constexpr int kNE6 = 21 + 6 + 2;
__global__ void grain_normal_k(FitFixed fx, const double *grains, const double *geo10, SpotList sp,
                               const int64_t *offsets, int64_t n_grains, double *ne) {
    // the thread's 29 accumulators in shared memory (column k of thread t at k * 128 + t), so one
    // pass carries all 6 tangents
    extern __shared__ double acc_s[];
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    for (int64_t gi = blockIdx.x; gi < n_grains; gi += gridDim.x) {
        for (int k = 0; k < kNE6; ++k) acc_s[k * 128 + t] = 0;
        const double *g6 = grains + 6 * gi;
        for (int64_t i = offsets[gi] + threadIdx.x; i < offsets[gi + 1]; i += blockDim.x) {
            double ru, rv, ju[6], jv[6];
            // spot left the detector: not part of this residual
            if (!spot_eval<6>(fx, 0, 0, g6, geo10, sp.iw[i], sp.ih[i], ru, rv, ju, jv)) continue;
            const double eu = ru - sp.uv[2 * i], ev = rv - sp.uv[2 * i + 1];
            int q = 0;
#pragma unroll
            for (int a = 0; a < 6; ++a)
#pragma unroll
                for (int b = a; b < 6; ++b) acc_s[(q++) * 128 + t] += ju[a] * ju[b] + jv[a] * jv[b];
#pragma unroll
            for (int a = 0; a < 6; ++a) acc_s[(21 + a) * 128 + t] += ju[a] * eu + jv[a] * ev;
            acc_s[27 * 128 + t] += eu * eu + ev * ev;
            acc_s[28 * 128 + t] += 1.0;
        }
        __syncthreads();
        for (int k = warp; k < kNE6; k += 4) {
            double v = acc_s[k * 128 + lane] + acc_s[k * 128 + lane + 32] + acc_s[k * 128 + lane + 64] +
                       acc_s[k * 128 + lane + 96];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
            if (lane == 0) ne[gi * kNE6 + k] = v;
        }
        __syncthreads();  // the next grain clears the accumulators
    }
}

// Cost (sum of squared residuals, spot count) of one grain per CTA for a parameter set.
__global__ void grain_cost_k(FitFixed fx, const double *grains, const double *geo10, SpotList sp,
                             const int64_t *offsets, int64_t n_grains, double *cost) {
    __shared__ double scratch[32 * 2];
    for (int64_t gi = blockIdx.x; gi < n_grains; gi += gridDim.x) {
        double acc[2] = {0, 0};
        const double *g6 = grains + 6 * gi;
        for (int64_t i = offsets[gi] + threadIdx.x; i < offsets[gi + 1]; i += blockDim.x) {
            double u, v;
            if (!spot_value(fx, g6, geo10, sp.iw[i], sp.ih[i], u, v)) {
                acc[0] += 1e6;  // a spot that leaves the detector counts as a large residual
                acc[1] += 1.0;
                continue;
            }
            const double eu = u - sp.uv[2 * i], ev = v - sp.uv[2 * i + 1];
            acc[0] += eu * eu + ev * ev;
            acc[1] += 1.0;
        }
        block_sum<2>(acc, scratch);
        if (threadIdx.x == 0) {
            cost[2 * gi] = acc[0];
            cost[2 * gi + 1] = acc[1];
        }
    }
}

// RMS distance of predicted spots between two parameter sets (fit vs ground truth), per grain.
__global__ void grain_rms_k(FitFixed fx, const double *grains, const double *truth, const double *geo10,
                            SpotList sp, const int64_t *offsets, int64_t n_grains, double *rms) {
    __shared__ double scratch[32 * 2];
    for (int64_t gi = blockIdx.x; gi < n_grains; gi += gridDim.x) {
        double acc[2] = {0, 0};
        for (int64_t i = offsets[gi] + threadIdx.x; i < offsets[gi + 1]; i += blockDim.x) {
            double u, v, ut, vt;
            const bool a = spot_value(fx, grains + 6 * gi, geo10, sp.iw[i], sp.ih[i], u, v);
            const bool b = spot_value(fx, truth + 6 * gi, geo10, sp.iw[i], sp.ih[i], ut, vt);
            if (!(a && b)) continue;
            acc[0] += (u - ut) * (u - ut) + (v - vt) * (v - vt);
            acc[1] += 1.0;
        }
        block_sum<2>(acc, scratch);
        if (threadIdx.x == 0) rms[gi] = acc[1] > 0 ? sqrt(acc[0] / acc[1]) : CUDART_INF;
    }
}

// Cholesky solve of (A + lambda*diag(A)) x = -b for an n x n SPD matrix stored as the upper
// triangle (row-major packing); returns false when the factorisation fails.
template <int N>
__device__ bool lm_solve(const double *upper, const double *b, double lambda, double *x) {
    double M[N][N];
    int q = 0;
    for (int a = 0; a < N; ++a)
        for (int c = a; c < N; ++c) {
            M[a][c] = upper[q];
            M[c][a] = upper[q];
            ++q;
        }
    for (int a = 0; a < N; ++a) M[a][a] *= (1.0 + lambda);
    for (int j = 0; j < N; ++j) {
        double d = M[j][j];
        for (int k = 0; k < j; ++k) d -= M[j][k] * M[j][k];
        if (!(d > 0)) return false;
        d = sqrt(d);
        M[j][j] = d;
        for (int i = j + 1; i < N; ++i) {
            double t = M[i][j];
            for (int k = 0; k < j; ++k) t -= M[i][k] * M[j][k];
            M[i][j] = t / d;
        }
    }
    double y[N];
    for (int i = 0; i < N; ++i) {
        double t = -b[i];
        for (int k = 0; k < i; ++k) t -= M[i][k] * y[k];
        y[i] = t / M[i][i];
    }
    for (int i = N - 1; i >= 0; --i) {
        double t = y[i];
        for (int k = i + 1; k < N; ++k) t -= M[k][i] * x[k];
        x[i] = t / M[i][i];
    }
    return true;
}

// Levenberg-Marquardt proposal per grain: trial = params + step.
__global__ void grain_lm_propose_k(const double *grains, const double *ne, const double *lambda, int64_t n,
                                   double *trial) {
    for (int64_t gi = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; gi < n; gi += (int64_t)gridDim.x * blockDim.x) {
        double x[6] = {0, 0, 0, 0, 0, 0};
        const double *e = ne + gi * kNE6;
        const bool ok = e[28] >= 6 && lm_solve<6>(e, e + 21, lambda[gi], x);
        for (int k = 0; k < 6; ++k) trial[6 * gi + k] = grains[6 * gi + k] + (ok ? x[k] : 0.0);
    }
}

// Accept the trial where it lowers the cost (lambda /= 10), else keep the point (lambda *= 10).
__global__ void grain_lm_accept_k(double *grains, const double *trial, const double *cost_now,
                                  const double *cost_trial, double *lambda, int64_t n, int *improved) {
    for (int64_t gi = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; gi < n; gi += (int64_t)gridDim.x * blockDim.x) {
        if (cost_trial[2 * gi] < cost_now[2 * gi]) {
            for (int k = 0; k < 6; ++k) grains[6 * gi + k] = trial[6 * gi + k];
            lambda[gi] = fmax(lambda[gi] * 0.1, 1e-9);
            if (cost_now[2 * gi] - cost_trial[2 * gi] > 1e-9 * cost_now[2 * gi]) atomicAdd(improved, 1);
        } else {
            lambda[gi] = fmin(lambda[gi] * 10.0, 1e9);
        }
    }
}

// ---- forward-only baseline: batched Nelder-Mead (fminsearchbnd) ----------------------------
// One CTA per grain.  Parameters live in the sine-transformed space of fminsearchbnd.m:263-265
// (x = lb + (ub - lb)(sin(z) + 1)/2); the simplex follows the standard Nelder-Mead moves
// (reflection 1, expansion 2, contraction 0.5, shrink 0.5; Lagarias et al. 1998 as used by
// fminsearch).  Every objective value is a cooperative sum over the grain's spots.
constexpr int kNM = 6;

__device__ double nm_objective(const FitFixed &fx, const double *geo10, const SpotList &sp, int64_t i0, int64_t i1,
                               const double *z, const double *lb, const double *ub, double *scratch) {
    double x[6];
    for (int k = 0; k < kNM; ++k) x[k] = lb[k] + (ub[k] - lb[k]) * (sin(z[k]) + 1.0) * 0.5;
    double acc[1] = {0};
    for (int64_t i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
        double u, v;
        if (!spot_value(fx, x, geo10, sp.iw[i], sp.ih[i], u, v)) {
            acc[0] += 1e6;
            continue;
        }
        const double eu = u - sp.uv[2 * i], ev = v - sp.uv[2 * i + 1];
        acc[0] += eu * eu + ev * ev;
    }
    block_sum<1>(acc, scratch);
    __shared__ double s_out;
    if (threadIdx.x == 0) s_out = acc[0];
    __syncthreads();
    const double r = s_out;
    __syncthreads();
    return r;
}

__global__ void grain_nm_k(FitFixed fx, double *grains, const double *geo10, SpotList sp, const int64_t *offsets,
                           int64_t n_grains, const double *half_width, int max_evals, int checkpoint, double *trace,
                           int n_ck) {
    __shared__ double scratch[32];
    __shared__ double simplex[kNM + 1][kNM], fval[kNM + 1];
    __shared__ double lb[kNM], ub[kNM], zr[kNM], ze[kNM], zc[kNM], cen[kNM];
    __shared__ int s_order[kNM + 1];
    for (int64_t gi = blockIdx.x; gi < n_grains; gi += gridDim.x) {
        const int64_t i0 = offsets[gi], i1 = offsets[gi + 1];
        if (threadIdx.x < kNM) {
            const double x0 = grains[6 * gi + threadIdx.x];
            lb[threadIdx.x] = x0 - half_width[threadIdx.x];
            ub[threadIdx.x] = x0 + half_width[threadIdx.x];
        }
        __syncthreads();
        // initial simplex in z-space: start at the centre (z = 0), fminsearch's 5% steps
        if (threadIdx.x == 0)
            for (int v = 0; v <= kNM; ++v)
                for (int k = 0; k < kNM; ++k) simplex[v][k] = (v == k + 1) ? 0.05 * 1.5707963267948966 : 0.0;
        __syncthreads();
        int evals = 0, ck = 0;
        for (int v = 0; v <= kNM; ++v) {
            const double f = nm_objective(fx, geo10, sp, i0, i1, simplex[v], lb, ub, scratch);
            if (threadIdx.x == 0) fval[v] = f;
            ++evals;
        }
        __syncthreads();
        while (evals < max_evals) {
            if (threadIdx.x == 0) {
                for (int v = 0; v <= kNM; ++v) s_order[v] = v;
                for (int a = 1; a <= kNM; ++a)
                    for (int b = a; b > 0 && fval[s_order[b]] < fval[s_order[b - 1]]; --b) {
                        const int t = s_order[b];
                        s_order[b] = s_order[b - 1];
                        s_order[b - 1] = t;
                    }
                for (int k = 0; k < kNM; ++k) {
                    double t = 0;
                    for (int v = 0; v < kNM; ++v) t += simplex[s_order[v]][k];
                    cen[k] = t / kNM;
                    zr[k] = 2.0 * cen[k] - simplex[s_order[kNM]][k];
                }
            }
            __syncthreads();
            const double fr = nm_objective(fx, geo10, sp, i0, i1, zr, lb, ub, scratch);
            ++evals;
            const int best = s_order[0], worst = s_order[kNM], second = s_order[kNM - 1];
            if (fr < fval[best]) {
                if (threadIdx.x == 0)
                    for (int k = 0; k < kNM; ++k) ze[k] = 3.0 * cen[k] - 2.0 * simplex[worst][k];
                __syncthreads();
                const double fe = nm_objective(fx, geo10, sp, i0, i1, ze, lb, ub, scratch);
                ++evals;
                if (threadIdx.x == 0) {
                    const double *src = fe < fr ? ze : zr;
                    for (int k = 0; k < kNM; ++k) simplex[worst][k] = src[k];
                    fval[worst] = fe < fr ? fe : fr;
                }
            } else if (fr < fval[second]) {
                if (threadIdx.x == 0) {
                    for (int k = 0; k < kNM; ++k) simplex[worst][k] = zr[k];
                    fval[worst] = fr;
                }
            } else {
                const bool outside = fr < fval[worst];
                if (threadIdx.x == 0)
                    for (int k = 0; k < kNM; ++k)
                        zc[k] = outside ? 1.5 * cen[k] - 0.5 * simplex[worst][k] : 0.5 * cen[k] + 0.5 * simplex[worst][k];
                __syncthreads();
                const double fc = nm_objective(fx, geo10, sp, i0, i1, zc, lb, ub, scratch);
                ++evals;
                if (fc < (outside ? fr : fval[worst])) {
                    if (threadIdx.x == 0) {
                        for (int k = 0; k < kNM; ++k) simplex[worst][k] = zc[k];
                        fval[worst] = fc;
                    }
                } else {
                    for (int v = 1; v <= kNM; ++v) {  // shrink towards the best vertex
                        const int vi = s_order[v];
                        if (threadIdx.x == 0)
                            for (int k = 0; k < kNM; ++k) simplex[vi][k] = simplex[best][k] + 0.5 * (simplex[vi][k] - simplex[best][k]);
                        __syncthreads();
                        const double f = nm_objective(fx, geo10, sp, i0, i1, simplex[vi], lb, ub, scratch);
                        ++evals;
                        if (threadIdx.x == 0) fval[vi] = f;
                    }
                }
            }
            __syncthreads();
            // checkpoint: best vertex in parameter space every `checkpoint` evaluations
            while (trace && ck < n_ck && evals >= (ck + 1) * checkpoint) {
                if (threadIdx.x == 0) {
                    int b = 0;
                    for (int v = 1; v <= kNM; ++v)
                        if (fval[v] < fval[b]) b = v;
                    for (int k = 0; k < kNM; ++k)
                        trace[((int64_t)ck * n_grains + gi) * 6 + k] =
                            lb[k] + (ub[k] - lb[k]) * (sin(simplex[b][k]) + 1.0) * 0.5;
                }
                ++ck;
            }
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            int b = 0;
            for (int v = 1; v <= kNM; ++v)
                if (fval[v] < fval[b]) b = v;
            for (int k = 0; k < kNM; ++k) grains[6 * gi + k] = lb[k] + (ub[k] - lb[k]) * (sin(simplex[b][k]) + 1.0) * 0.5;
            for (; trace && ck < n_ck; ++ck)
                for (int k = 0; k < kNM; ++k) trace[((int64_t)ck * n_grains + gi) * 6 + k] = grains[6 * gi + k];
        }
        __syncthreads();
    }
}

// ---- geometry fit: normal equations of every start ------------------------------------
// Spots are split across CTAs (blockIdx.x) for start blockIdx.y; partial sums are added
// atomically into the start's 67 accumulators (55 upper J^T J, 10 J^T r, r^T r, n).
constexpr int kNE10 = 55 + 10 + 2;
__global__ void geo_normal_k(FitFixed fx, const double *grains, const double *starts, SpotList sp, double *ne) {
    // Each thread's 67 accumulators live in shared memory (column k of thread t at k * 128 + t),
    // which leaves the registers to one pass of all 10 tangent directions: against 67 register
    // accumulators and five passes of 2 tangents, an LM iteration of the 64-start Al fit runs
    // 2.5x faster (0.132 s against 0.331 s to 0.1 px).
    extern __shared__ double acc_s[];
    const int st = blockIdx.y, t = threadIdx.x;
    const double *geo = starts + 10 * st;
    for (int k = 0; k < kNE10; ++k) acc_s[k * 128 + t] = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < sp.n; i += (int64_t)gridDim.x * blockDim.x) {
        double ju[10], jv[10], ru = 0, rv = 0;
        const double *g6 = grains + 6 * (int64_t)sp.grain[i];
        if (!spot_eval<10>(fx, 1, 0, g6, geo, sp.iw[i], sp.ih[i], ru, rv, ju, jv)) continue;
        const double eu = ru - sp.uv[2 * i], ev = rv - sp.uv[2 * i + 1];
        int q = 0;
#pragma unroll
        for (int a = 0; a < 10; ++a)
#pragma unroll
            for (int b = a; b < 10; ++b) acc_s[(q++) * 128 + t] += ju[a] * ju[b] + jv[a] * jv[b];
#pragma unroll
        for (int a = 0; a < 10; ++a) acc_s[(55 + a) * 128 + t] += ju[a] * eu + jv[a] * ev;
        acc_s[65 * 128 + t] += eu * eu + ev * ev;
        acc_s[66 * 128 + t] += 1.0;
    }
    __syncthreads();
    // column sums: warp w sums columns w, w + 4, ...
    const int lane = t & 31, warp = t >> 5;
    for (int k = warp; k < kNE10; k += 4) {
        double v = acc_s[k * 128 + lane] + acc_s[k * 128 + lane + 32] + acc_s[k * 128 + lane + 64] +
                   acc_s[k * 128 + lane + 96];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) atomicAdd(&ne[st * kNE10 + k], v);
    }
}

__global__ void geo_cost_k(FitFixed fx, const double *grains, const double *starts, SpotList sp, double *cost) {
    __shared__ double scratch[32 * 2];
    const int st = blockIdx.y;
    const double *geo = starts + 10 * st;
    double acc[2] = {0, 0};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < sp.n; i += (int64_t)gridDim.x * blockDim.x) {
        double u, v;
        if (!spot_value(fx, grains + 6 * (int64_t)sp.grain[i], geo, sp.iw[i], sp.ih[i], u, v)) {
            acc[0] += 1e6;
            acc[1] += 1.0;
            continue;
        }
        const double eu = u - sp.uv[2 * i], ev = v - sp.uv[2 * i + 1];
        acc[0] += eu * eu + ev * ev;
        acc[1] += 1.0;
    }
    block_sum<2>(acc, scratch);
    if (threadIdx.x == 0) {
        atomicAdd(&cost[2 * st], acc[0]);
        atomicAdd(&cost[2 * st + 1], acc[1]);
    }
}

__global__ void geo_lm_propose_k(const double *starts, const double *ne, const double *lambda, int n,
                                 double *trial) {
    const int st = blockIdx.x * blockDim.x + threadIdx.x;
    if (st >= n) return;
    double x[10];
    for (int k = 0; k < 10; ++k) x[k] = 0;
    const double *e = ne + st * kNE10;
    const bool ok = e[66] >= 10 && lm_solve<10>(e, e + 55, lambda[st], x);
    for (int k = 0; k < 10; ++k) trial[10 * st + k] = starts[10 * st + k] + (ok ? x[k] : 0.0);
}

__global__ void geo_lm_accept_k(double *starts, const double *trial, const double *cost_now,
                                const double *cost_trial, double *lambda, int n, int *improved) {
    const int st = blockIdx.x * blockDim.x + threadIdx.x;
    if (st >= n) return;
    if (cost_trial[2 * st] < cost_now[2 * st]) {
        for (int k = 0; k < 10; ++k) starts[10 * st + k] = trial[10 * st + k];
        lambda[st] = fmax(lambda[st] * 0.1, 1e-9);
        if (cost_now[2 * st] - cost_trial[2 * st] > 1e-9 * cost_now[2 * st]) atomicAdd(improved, 1);
    } else {
        lambda[st] = fmin(lambda[st] * 10.0, 1e9);
    }
}

// RMS distance of predicted spots between each start's geometry and the true geometry.
__global__ void geo_rms_k(FitFixed fx, const double *grains, const double *starts, const double *truth,
                          SpotList sp, double *acc_out) {
    __shared__ double scratch[32 * 2];
    const int st = blockIdx.y;
    double acc[2] = {0, 0};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < sp.n; i += (int64_t)gridDim.x * blockDim.x) {
        double u, v, ut, vt;
        const double *g6 = grains + 6 * (int64_t)sp.grain[i];
        const bool a = spot_value(fx, g6, starts + 10 * st, sp.iw[i], sp.ih[i], u, v);
        const bool b = spot_value(fx, g6, truth, sp.iw[i], sp.ih[i], ut, vt);
        if (!(a && b)) continue;
        acc[0] += (u - ut) * (u - ut) + (v - vt) * (v - vt);
        acc[1] += 1.0;
    }
    block_sum<2>(acc, scratch);
    if (threadIdx.x == 0) {
        atomicAdd(&acc_out[2 * st], acc[0]);
        atomicAdd(&acc_out[2 * st + 1], acc[1]);
    }
}

// ---- synthetic measured spots ---------------------------------------------------------
// Count / fill the selected (omega, hkl) landings of every grain at the given geometry.
__global__ void spots_count_k(FitFixed fx, const double *grains, const double *geo10, int64_t n_grains,
                              int64_t *counts) {
    __shared__ int s_cnt;
    for (int64_t gi = blockIdx.x; gi < n_grains; gi += gridDim.x) {
        if (threadIdx.x == 0) s_cnt = 0;
        __syncthreads();
        int local = 0;
        for (int j = threadIdx.x; j < fx.nrot * fx.nhkl; j += blockDim.x) {
            double u, v;
            if (spot_value(fx, grains + 6 * gi, geo10, j / fx.nhkl, j % fx.nhkl, u, v, true)) ++local;
        }
        atomicAdd(&s_cnt, local);
        __syncthreads();
        if (threadIdx.x == 0) counts[gi] = s_cnt;
        __syncthreads();
    }
}

__global__ void spots_fill_k(FitFixed fx, const double *grains, const double *geo10, int64_t n_grains,
                             const int64_t *offsets, SpotList sp) {
    __shared__ int s_pos;
    for (int64_t gi = blockIdx.x; gi < n_grains; gi += gridDim.x) {
        if (threadIdx.x == 0) s_pos = 0;
        __syncthreads();
        // ordered fill: chunks of blockDim reflections, warp ballots + a block prefix
        for (int j0 = 0; j0 < fx.nrot * fx.nhkl; j0 += blockDim.x) {
            const int j = j0 + threadIdx.x;
            double u = 0, v = 0;
            const bool ok =
                j < fx.nrot * fx.nhkl && spot_value(fx, grains + 6 * gi, geo10, j / fx.nhkl, j % fx.nhkl, u, v, true);
            __shared__ int s_warp[32];
            const unsigned m = __ballot_sync(0xffffffffu, ok);
            const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
            if (lane == 0) s_warp[warp] = __popc(m);
            __syncthreads();
            int before = 0;
            for (int w = 0; w < warp; ++w) before += s_warp[w];
            if (ok) {
                const int64_t k = offsets[gi] + s_pos + before + __popc(m & ((1u << lane) - 1u));
                sp.grain[k] = (int32_t)gi;
                sp.iw[k] = j / fx.nhkl;
                sp.ih[k] = j % fx.nhkl;
                sp.uv[2 * k] = u;
                sp.uv[2 * k + 1] = v;
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                int tot = 0;
                for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += s_warp[w];
                s_pos += tot;
            }
            __syncthreads();
        }
    }
}

inline int grid_for(int64_t n, int per) {
    int64_t b = (n + per - 1) / per;
    if (b < 1) b = 1;
    if (b > 65535LL * 16) b = 65535LL * 16;
    return (int)b;
}

}  // namespace

cudaError_t fit_residual_jacobian(const FitFixed &fx, int mode, const double *grains, const double *geo10,
                                  const SpotList &sp, double *res, double *jac, cudaStream_t s) {
    residual_jac_k<2><<<grid_for(sp.n, 128), 128, 0, s>>>(fx, mode, grains, geo10, sp, res, jac);
    return cudaGetLastError();
}

cudaError_t fit_spots_count(const FitFixed &fx, const double *grains, const double *geo10, int64_t n_grains,
                            int64_t *counts, cudaStream_t s) {
    spots_count_k<<<grid_for(n_grains, 1), 256, 0, s>>>(fx, grains, geo10, n_grains, counts);
    return cudaGetLastError();
}

cudaError_t fit_spots_fill(const FitFixed &fx, const double *grains, const double *geo10, int64_t n_grains,
                           const int64_t *offsets, const SpotList &sp, cudaStream_t s) {
    spots_fill_k<<<grid_for(n_grains, 1), 256, 0, s>>>(fx, grains, geo10, n_grains, offsets, sp);
    return cudaGetLastError();
}

cudaError_t fit_grain_normal(const FitFixed &fx, const double *grains, const double *geo10, const SpotList &sp,
                             const int64_t *offsets, int64_t n_grains, double *ne, cudaStream_t s) {
    const size_t smem = sizeof(double) * kNE6 * 128;
    const cudaError_t e = allow_smem((const void *)grain_normal_k, smem);
    if (e != cudaSuccess) return e;
    grain_normal_k<<<grid_for(n_grains, 1), 128, smem, s>>>(fx, grains, geo10, sp, offsets, n_grains, ne);
    return cudaGetLastError();
}

cudaError_t fit_grain_cost(const FitFixed &fx, const double *grains, const double *geo10, const SpotList &sp,
                           const int64_t *offsets, int64_t n_grains, double *cost, cudaStream_t s) {
    grain_cost_k<<<grid_for(n_grains, 1), 128, 0, s>>>(fx, grains, geo10, sp, offsets, n_grains, cost);
    return cudaGetLastError();
}

cudaError_t fit_grain_rms(const FitFixed &fx, const double *grains, const double *truth, const double *geo10,
                          const SpotList &sp, const int64_t *offsets, int64_t n_grains, double *rms, cudaStream_t s) {
    grain_rms_k<<<grid_for(n_grains, 1), 128, 0, s>>>(fx, grains, truth, geo10, sp, offsets, n_grains, rms);
    return cudaGetLastError();
}

cudaError_t fit_grain_lm_propose(const double *grains, const double *ne, const double *lambda, int64_t n,
                                 double *trial, cudaStream_t s) {
    grain_lm_propose_k<<<grid_for(n, 128), 128, 0, s>>>(grains, ne, lambda, n, trial);
    return cudaGetLastError();
}

cudaError_t fit_grain_lm_accept(double *grains, const double *trial, const double *cost_now, const double *cost_trial,
                                double *lambda, int64_t n, int *improved, cudaStream_t s) {
    grain_lm_accept_k<<<grid_for(n, 128), 128, 0, s>>>(grains, trial, cost_now, cost_trial, lambda, n, improved);
    return cudaGetLastError();
}

cudaError_t fit_grain_nm(const FitFixed &fx, double *grains, const double *geo10, const SpotList &sp,
                         const int64_t *offsets, int64_t n_grains, const double *half_width, int max_evals,
                         int checkpoint, double *trace, int n_ck, cudaStream_t s) {
    grain_nm_k<<<grid_for(n_grains, 1), 128, 0, s>>>(fx, grains, geo10, sp, offsets, n_grains, half_width, max_evals,
                                                     checkpoint, trace, n_ck);
    return cudaGetLastError();
}

cudaError_t fit_geo_normal(const FitFixed &fx, const double *grains, const double *starts, int n_starts,
                           const SpotList &sp, double *ne, int num_sms, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(ne, 0, sizeof(double) * kNE10 * n_starts, s);
    if (e != cudaSuccess) return e;
    const int gx = grid_for(sp.n, 128) < num_sms * 4 ? grid_for(sp.n, 128) : num_sms * 4;
    const size_t smem = sizeof(double) * kNE10 * 128;
    e = allow_smem((const void *)geo_normal_k, smem);
    if (e != cudaSuccess) return e;
    geo_normal_k<<<dim3(gx, n_starts), 128, smem, s>>>(fx, grains, starts, sp, ne);
    return cudaGetLastError();
}

cudaError_t fit_geo_cost(const FitFixed &fx, const double *grains, const double *starts, int n_starts,
                         const SpotList &sp, double *cost, int num_sms, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(cost, 0, sizeof(double) * 2 * n_starts, s);
    if (e != cudaSuccess) return e;
    const int gx = grid_for(sp.n, 128) < num_sms * 4 ? grid_for(sp.n, 128) : num_sms * 4;
    geo_cost_k<<<dim3(gx, n_starts), 128, 0, s>>>(fx, grains, starts, sp, cost);
    return cudaGetLastError();
}

cudaError_t fit_geo_rms(const FitFixed &fx, const double *grains, const double *starts, int n_starts,
                        const double *truth, const SpotList &sp, double *acc, int num_sms, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(acc, 0, sizeof(double) * 2 * n_starts, s);
    if (e != cudaSuccess) return e;
    const int gx = grid_for(sp.n, 128) < num_sms * 4 ? grid_for(sp.n, 128) : num_sms * 4;
    geo_rms_k<<<dim3(gx, n_starts), 128, 0, s>>>(fx, grains, starts, truth, sp, acc);
    return cudaGetLastError();
}

cudaError_t fit_geo_lm_propose(const double *starts, const double *ne, const double *lambda, int n, double *trial,
                               cudaStream_t s) {
    geo_lm_propose_k<<<(n + 63) / 64, 64, 0, s>>>(starts, ne, lambda, n, trial);
    return cudaGetLastError();
}

cudaError_t fit_geo_lm_accept(double *starts, const double *trial, const double *cost_now, const double *cost_trial,
                              double *lambda, int n, int *improved, cudaStream_t s) {
    geo_lm_accept_k<<<(n + 63) / 64, 64, 0, s>>>(starts, trial, cost_now, cost_trial, lambda, n, improved);
    return cudaGetLastError();
}

}  // namespace grc
