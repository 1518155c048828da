// grc_chain.cuh -- the per-reflection chain of forward_comp.m shared by the scoring kernels:
// FP64 constants of one (voxel, omega) pair, their FP32 row, the FP64 landing (the exact path)
// and the FP32 landing with its ambiguity band, and the FP32 Gw / window of one reflection.
// Included by grc_score.cu and grc_scan.cu; every function is device-inline.
#pragma once
#include <cuda_runtime.h>
#include <math_constants.h>
#include <stdint.h>

#include "grc_internal.h"

namespace grc {
namespace {

constexpr unsigned kFull = 0xffffffffu;

// FP64 constants of one (voxel, omega) pair, forward_comp.m:17-26,42,51.
struct OmegaRow {
    double kx, ky, kz, L2;  // unit incident direction (lab), L2 of forward_comp.m:42
    double ax, ay, az, num; // center - SamposW; t-numerator of forward_comp.m:51
    double r2d, r3d, c, s;  // RotDet(:,2).d, RotDet(:,3).d with d = SamposW - D0; cos/sin omega
};

// The same row for the FP32 chain, kept in shared memory: the terms that do not depend on
// the reflection are folded in (RotDet(1,:) * ax and the pixel scale), plus
// k_w = Omega^T k_in for the prefilter.
struct __align__(16) RowF {
    float cN, ky, kz, L2;   // cN = R(1,1) ax
    float cY, ay, az, num;  // cY = R(1,2) ax / pxy
    float u0, v0, c, s;     // u0 = dety0 - r2d / pxy, v0 = detz0 - r3d / pxz
    float wx, wy, wz, cZ;   // k_w; cZ = R(1,3) ax / pxz
};
static_assert(sizeof(RowF) == 64, "RowF layout");

// Pixel-rounding ambiguity band of the FP32 landing chain.  Its error against the
// FP64 chain stays below 1.4e-3 px on the 1024^2 / 2048^2 geometries (measured over
// 3.4e5 landings); landings closer than this to a half-pixel boundary are recomputed
// in FP64, so every decision equals the FP64 one.  A build with -DGRC_AUDIT re-decides
// every FP32 decision in FP64 (CTA sweep): at 0.003 px it found no disagreement in
// 1.72e10 decisions (FCC Al 2048^2 x 361 and BCC Fe 1024^2 x 181 scans, 64 seeds x 32,768
// orientations each), at 0.001 px two in 1.7e9; the band keeps a third above the audited
// 0.003 px.
#ifndef GRC_AMBIG_PX
#define GRC_AMBIG_PX 0.004f
#endif
constexpr float kAmbigPx = GRC_AMBIG_PX;

__device__ __forceinline__ size_t align16(size_t x) { return (x + 15) & ~size_t(15); }

__device__ __forceinline__ OmegaRow omega_row(const Geo &g, const double2 cs, const double *__restrict__ vp) {
    const double px = vp[0], py = vp[1] - g.rao, pz = vp[2];
    const double spx = g.S[0] * px + g.S[1] * py + g.S[2] * pz;
    const double spy = g.S[3] * px + g.S[4] * py + g.S[5] * pz;
    const double spz = g.S[6] * px + g.S[7] * py + g.S[8] * pz;
    const double L = g.lss + g.lsd;
    const double c = cs.x, s = cs.y;
    const double swx = c * spx - s * spy, swy = s * spx + c * spy, swz = spz;
    const double gx = g.lss + swx, gy = swy - g.p0y + g.rao, gz = swz - g.p0z;
    const double ngp = sqrt(gx * gx + gy * gy + gz * gz);
    OmegaRow r;
    r.kx = gx / ngp;
    r.ky = gy / ngp;
    r.kz = gz / ngp;
    r.L2 = (g.lsd - swx) * ngp / gx;  // (Lsd - SamposW_x) / cos(alpha)
    r.ax = g.lsd - swx;
    r.ay = gy * L / gx - swy;
    r.az = gz * L / gx - swz;
    const double dx = swx - g.lsd, dy = swy - g.dety00 + g.rao, dz = swz - g.detz00;
    r.num = -(g.R[0] * dx + g.R[3] * dy + g.R[6] * dz);
    r.r2d = g.R[1] * dx + g.R[4] * dy + g.R[7] * dz;
    r.r3d = g.R[2] * dx + g.R[5] * dy + g.R[8] * dz;
    r.c = c;
    r.s = s;
    return r;
}

// FP32 row from the FP64 one (the folded constants are formed in FP64 and rounded once).
__device__ __forceinline__ RowF row_f32(const Geo &g, const OmegaRow &r) {
    RowF f;
    f.cN = (float)(g.R[0] * r.ax);
    f.ky = (float)r.ky; f.kz = (float)r.kz; f.L2 = (float)r.L2;
    f.cY = (float)(g.R[1] * r.ax / g.pxy);
    f.ay = (float)r.ay; f.az = (float)r.az; f.num = (float)r.num;
    f.u0 = (float)(g.dety0 - r.r2d / g.pxy);
    f.v0 = (float)(g.detz0 - r.r3d / g.pxz);
    f.c = (float)r.c; f.s = (float)r.s;
    f.wx = (float)(r.c * r.kx + r.s * r.ky);
    f.wy = (float)(-r.s * r.kx + r.c * r.ky);
    f.wz = (float)r.kz;
    f.cZ = (float)(g.R[2] * r.ax / g.pxz);
    return f;
}

// Omega table of one voxel in shared memory (all threads of the CTA).
__device__ void build_rows(const Geo &g, const double2 *__restrict__ rot_cs, const double *__restrict__ vp,
                           RowF *rows) {
    for (int iw = threadIdx.x; iw < g.nrot; iw += blockDim.x) rows[iw] = row_f32(g, omega_row(g, rot_cs[iw], vp));
}

// SUB = S*U*B (FP64, 9 values) of one trial.
__device__ __forceinline__ void sub_matrix(const Geo &g, const double *__restrict__ U, double *SUB) {
    double SU[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            SU[3 * i + j] = g.S[3 * i] * U[j] + g.S[3 * i + 1] * U[3 + j] + g.S[3 * i + 2] * U[6 + j];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            SUB[3 * i + j] = SU[3 * i] * g.B[j] + SU[3 * i + 1] * g.B[3 + j] + SU[3 * i + 2] * g.B[6 + j];
}

// Gw = S*U*B*h and |Gw| (forward_comp.m:15-16): FP32 table in shared memory plus the
// FP64 SUB matrix kept for the exact recomputation of ambiguous reflections.
__device__ __forceinline__ float4 window_of(const Geo &g, float G_f);

__device__ void build_gw(const Geo &g, const double *__restrict__ hkl, const double *__restrict__ U, float4 *gw,
                         float4 *win, double *sub) {
    const int ih = threadIdx.x;
    if (ih >= g.nhkl && ih >= 9) return;
    double SUB[9];
    sub_matrix(g, U, SUB);
    if (ih < 9) sub[ih] = SUB[ih];  // threads 0..8 write SUB even when nhkl < 9
    if (ih >= g.nhkl) return;
    const double h = hkl[3 * ih], k = hkl[3 * ih + 1], l = hkl[3 * ih + 2];
    const double x = SUB[0] * h + SUB[1] * k + SUB[2] * l;
    const double y = SUB[3] * h + SUB[4] * k + SUB[5] * l;
    const double z = SUB[6] * h + SUB[7] * k + SUB[8] * l;
    const double Gd = sqrt(x * x + y * y + z * z);
    gw[ih] = make_float4((float)x, (float)y, (float)z, (float)(1.0 / Gd));
    win[ih] = window_of(g, (float)Gd);
}

// Exact FP64 evaluation of one reflection: the linear map index of its pixel, or -1
// when select3 of forward_comp.m:61-65 rejects it.  Algebraic form of
// forward_comp.m:28-59: sin(theta) = -cos(beta), cos(theta) = sin(beta), sin(phiy)
// expanded, and the ray/plane intersection without normalising K_out.
__device__ __forceinline__ int64_t landing_fp64(const Geo &g, const OmegaRow &r, double gxw, double gyw,
                                                double gzw, int iw, double *lam_out = nullptr) {
    const double G = sqrt(gxw * gxw + gyw * gyw + gzw * gzw);
    const double Gtx = r.c * gxw - r.s * gyw, Gty = r.s * gxw + r.c * gyw, Gtz = gzw;
    const double x = (r.kx * Gtx + r.ky * Gty + r.kz * Gtz) / G;  // cos(beta)
    const double lam = 2.0 * (2.0 * CUDART_PI / G) * (-x);        // 2 d sin(theta)
    if (lam_out) *lam_out = lam;
    if (!(x < 0.0 && x > g.cbmax && lam > g.lmin && lam < g.lmax)) return -1;
    const double st = -x, ct = sqrt(1.0 - x * x);
    const double s2 = 2.0 * st * ct, c2 = 1.0 - 2.0 * st * st;
    const double konst = sqrt(Gty * Gty + Gtz * Gtz);
    const double gy = Gty / konst, gz = Gtz / konst;
    const double cphx = gy * r.ky + gz * r.kz;
    const double sphx = sqrt(fmax(0.0, 1.0 - cphx * cphx));
    const double sphy = sphx * c2 - cphx * s2;
    const double diff = r.L2 * s2 / sphy;
    const double Kx = r.ax, Ky = r.ay + diff * gy, Kz = r.az + diff * gz;
    const double nK = g.R[0] * Kx + g.R[3] * Ky + g.R[6] * Kz;
    const double f = r.num / nK;
    const double y2 = f * (g.R[1] * Kx + g.R[4] * Ky + g.R[7] * Kz) + r.r2d;
    const double z2 = f * (g.R[2] * Kx + g.R[5] * Ky + g.R[8] * Kz) + r.r3d;
    const double u = g.dety0 - y2 / g.pxy, v = g.detz0 - z2 / g.pxz;
    // 1 <= round(u) <= detysize  <=>  0.5 <= u < detysize + 0.5 (round half away from zero)
    if (!(u >= 0.5 && u < g.detysize + 0.5 && v >= 0.5 && v < g.detzsize + 0.5)) return -1;
    const double ru = round(u), rv = round(v);
    if (ru >= g.bsy0 && ru <= g.bsy1 && rv >= g.bsz0 && rv <= g.bsz1) return -1;
    return (int64_t)iw * g.plane + (int64_t)(ru - 1.0) * g.detzsize + (int64_t)(rv - 1.0);
}

// The exact path for one ambiguous item: FP64 omega row and Gw rebuilt from the inputs.
// Kept out of line (rarely taken) and reads the geometry from its global-memory copy.
__device__ __noinline__ int64_t landing_exact(const Geo *__restrict__ gd, const double2 *__restrict__ rot_cs,
                                              const double *__restrict__ vp, const double *__restrict__ hkl,
                                              const double *sub, int iw, int ih) {
    const Geo &g = *gd;
    const OmegaRow r = omega_row(g, rot_cs[iw], vp);
    const double h = hkl[3 * ih], k = hkl[3 * ih + 1], l = hkl[3 * ih + 2];
    const double x = sub[0] * h + sub[1] * k + sub[2] * l;
    const double y = sub[3] * h + sub[4] * k + sub[5] * l;
    const double z = sub[6] * h + sub[7] * k + sub[8] * l;
    return landing_fp64(g, r, x, y, z, iw);
}

// Window thresholds of one reflection on t = -(k_w . Gw) = |G|^2 lambda / (4 pi):
// lambda in (lambda_min, lambda_max) and cos(beta) > cos(beta_max).  Returned as
// (lo, hi) = the interval widened by the FP32 margin (prefilter) and (lo_in, hi_in)
// = narrowed by it (inside, the FP32 decision is certain).
__device__ __forceinline__ float4 window_of(const Geo &g, float G_f) {
    const double G = G_f, G2 = G * G;
    const double inv4pi = 0.25 / CUDART_PI;
    double lo = g.lmin * G2 * inv4pi, hi = g.lmax * G2 * inv4pi;
    if (g.cbmax > -1.0) hi = fmin(hi, -g.cbmax * G);
    lo = fmax(lo, 0.0);
    const double m = 1e-5 * G;  // >> FP32 error of k_w . G (~4e-7 |G|)
    return make_float4((float)(lo - m), (float)(hi + m), (float)(lo + m), (float)(hi - m));
}

// FP32 landing chain (the algebra of landing_fp64 with the row's constant terms folded in).
// Returns the in-plane map offset (dety-1)*detzsize + (detz-1), -1 for a certain rejection,
// or -2 when the item lies within the ambiguity band of a decision boundary and must be
// decided by landing_exact.
__device__ __forceinline__ int landing_fp32(const Geo &g, const RowF &r, const float4 gw, float lo_in, float hi_in) {
    // k_in . (Omega Gw) = (Omega^T k_in) . Gw: the prefilter's product, without rotating G
    const float dot = r.wx * gw.x + r.wy * gw.y + r.wz * gw.z;
    const float t = -dot;
    if (!(t > lo_in && t < hi_in)) return -2;  // near the wavelength / Bragg-angle window edge
    const float Gty = r.s * gw.x + r.c * gw.y, Gtz = gw.z;
    // gw.w holds 1/|G|; reciprocal and square-root intrinsics (a few ulp) stay far inside
    // the ambiguity band
    const float x = dot * gw.w;
    const float q = fmaxf(1.0f - x * x, 0.0f);
    const float st = -x, ct = q * rsqrtf(q);
    const float s2 = 2.0f * st * ct, c2 = 1.0f - 2.0f * st * st;
    const float rk = rsqrtf(Gty * Gty + Gtz * Gtz);
    const float gy = Gty * rk, gz = Gtz * rk;
    const float cphx = gy * r.ky + gz * r.kz;
    const float p = fmaxf(1.0f - cphx * cphx, 0.0f);
    const float sphx = p * rsqrtf(p);
    const float sphy = sphx * c2 - cphx * s2;
    const float diff = __fdividef(r.L2 * s2, sphy);
    const float Ky = r.ay + diff * gy, Kz = r.az + diff * gz;  // K_x = ax lives in cN, cY, cZ
    const float nK = r.cN + g.Rf[3] * Ky + g.Rf[6] * Kz;
    const float f = __fdividef(r.num, nK);
    const float u = r.u0 - f * (r.cY + g.Ruf[0] * Ky + g.Ruf[1] * Kz);
    const float v = r.v0 - f * (r.cZ + g.Rvf[0] * Ky + g.Rvf[1] * Kz);
    if (!(fabsf(u) < 2e6f && fabsf(v) < 2e6f)) {  // detectors have at most 10^6 pixels per side
        // far off the detector (or NaN): certain rejection only for finite values
        return (isfinite(u) && isfinite(v)) ? -1 : -2;
    }
    // nearest integer by the 1.5*2^23 addition (|u|, |v| < 2^22 here): the sum's low mantissa
    // bits hold the rounded value, read back as an integer without a conversion instruction.
    // Within the ambiguity band of a half-pixel the item goes to the exact path, so the tie
    // rule of the rounding never decides anything.
    constexpr float kRound = 12582912.0f;
    const float tu = __fadd_rn(u, kRound), tv = __fadd_rn(v, kRound);
    const float ru = __fsub_rn(tu, kRound), rv = __fsub_rn(tv, kRound);
    if (fabsf(u - ru) > 0.5f - kAmbigPx || fabsf(v - rv) > 0.5f - kAmbigPx) return -2;
    const int iu = __float_as_int(tu) - 0x4B400000, iv = __float_as_int(tv) - 0x4B400000;
    if (!(iu >= 1 && iu <= g.detysize && iv >= 1 && iv <= g.detzsize)) return -1;
    if (ru >= g.bsy0f && ru <= g.bsy1f && rv >= g.bsz0f && rv <= g.bsz1f) return -1;
    return (int)((uint32_t)(iu - 1) * (uint32_t)g.detzsize + (uint32_t)(iv - 1));  // < 2^31 pixels per plane
}

// Gw (FP32) of one reflection from the slot's S*U*B and h; .w = 1/|Gw|.
__device__ __forceinline__ float4 gw_of(const float *sf, const float4 h) {
    const float x = sf[0] * h.x + sf[1] * h.y + sf[2] * h.z;
    const float y = sf[3] * h.x + sf[4] * h.y + sf[5] * h.z;
    const float z = sf[6] * h.x + sf[7] * h.y + sf[8] * h.z;
    return make_float4(x, y, z, rsqrtf(x * x + y * y + z * z));
}

// Window on t = -(k_w . Gw) in FP32 (see window_of) from rG = 1/|G|; the 1e-5 |G|
// margins dominate its FP32 rounding.
__device__ __forceinline__ float4 window_f(const Geo &g, const float4 gv) {
    const float G2 = gv.x * gv.x + gv.y * gv.y + gv.z * gv.z, G = G2 * gv.w;
    float lo = g.lo4pif * G2, hi = g.hi4pif * G2;
    if (g.cbmaxf > -1.0f) hi = fminf(hi, -g.cbmaxf * G);
    lo = fmaxf(lo, 0.0f);
    const float m = 1e-5f * G;
    return make_float4(lo - m, hi + m, lo + m, hi - m);
}

// Result of one trial from its 8-bit code histogram (256 u16 bins in 128 words; bin 255 counts the
// saturated codes >= 255), by one warp: Nr_simu = the total, Nr_intersect = the total below n_hit
// (< 255), and the exact median when both middle ranks fall below the saturated bin; otherwise
// the median is left NaN and the trial is listed for the radix refine pass.
__device__ __forceinline__ void hist8_finish(const Geo &g, const ScoreBufs &b, const uint32_t *h, int64_t t) {
    constexpr unsigned kAll = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    // lane owns bins [8*lane, 8*lane+8)
    uint32_t bins[8];
    uint32_t local = 0, hits = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const uint32_t wv = h[4 * lane + i];
        bins[2 * i] = wv & 0xffffu;
        bins[2 * i + 1] = wv >> 16;
    }
    const uint32_t sat = __shfl_sync(kAll, bins[7], 31);  // bin 255: saturated codes (>= 255)
    if (lane == 31) bins[7] = 0;  // not part of the exact range
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        local += bins[i];
        if ((uint32_t)(8 * lane + i) < g.n_hit) hits += bins[i];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) hits += __shfl_xor_sync(kAll, hits, o);
    uint32_t incl = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(kAll, incl, o);
        if (lane >= o) incl += y;
    }
    const uint32_t inr = __shfl_sync(kAll, incl, 31);
    const int n = (int)(inr + sat), inter = (int)hits;  // Nr_simu, Nr_intersect
    const uint32_t excl = incl - local;
    const uint32_t ra = (uint32_t)(n + 1) / 2, rb = (uint32_t)n / 2 + 1;
    int ca = -1, cb = -1;
    if (n > 0 && rb <= inr) {
        uint32_t cum = excl;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            if (ca < 0 && cum < ra && ra <= cum + bins[i]) ca = 8 * lane + i;
            if (cb < 0 && cum < rb && rb <= cum + bins[i]) cb = 8 * lane + i;
            cum += bins[i];
        }
    }
    const unsigned ma = __ballot_sync(kAll, ca >= 0), mb = __ballot_sync(kAll, cb >= 0);
    ca = ma ? __shfl_sync(kAll, ca, __ffs(ma) - 1) : -1;
    cb = mb ? __shfl_sync(kAll, cb, __ffs(mb) - 1) : -1;
    if (lane == 0) {
        TrialRes r;
        r.simu = n;
        r.inter = inter;
        if (n == 0) {
            r.median = 2000.0;  // forward_comp.m:89
        } else if (ca >= 0 && cb >= 0) {
            r.median = ((double)b.vals[ca] + (double)b.vals[cb]) / 2.0;
        } else {
            r.median = CUDART_NAN;
            const int k = atomicAdd(b.work_counter + 4, 1);
            b.refine_list[k] = t;
        }
        b.res[t] = r;
    }
}

// First-maximum key of a trial's completeness within its group: larger completeness wins, NaN
// (0/0) loses to every number, and among equal values the smaller index in the group wins
// (MATLAB max: first maximum, NaN ignored; all NaN gives the first index).
__device__ __forceinline__ unsigned long long group_key_of(int simu, int inter, int64_t index_in_group) {
    const float C = (float)((double)inter / (double)simu);  // the epilogue's completeness
    const uint32_t hi = isnan(C) ? 0u : __float_as_uint(C) + 1u;
    const uint32_t lo = 0xffffffffu - (uint32_t)index_in_group;
    return ((unsigned long long)hi << 32) | lo;
}

__device__ __forceinline__ unsigned long long shfl_xor_u64(unsigned long long v, int o) {
    const uint32_t lo = __shfl_xor_sync(0xffffffffu, (uint32_t)v, o);
    const uint32_t hi = __shfl_xor_sync(0xffffffffu, (uint32_t)(v >> 32), o);
    return ((unsigned long long)hi << 32) | lo;
}

// Folds the keys of a warp's trials (trial t of lane, `in` = lane holds one) into b.group_key:
// one atomic per warp when all its trials share a group, else one per trial.
__device__ __forceinline__ void fold_group_key(const ScoreBufs &b, bool in, int64_t t, int simu, int inter) {
    const int64_t gs = b.group_size;
    const int64_t grp = in ? t / gs : -1;
    unsigned long long key = in ? group_key_of(simu, inter, t - grp * gs) : 0ull;
    const int64_t g0 = __shfl_sync(0xffffffffu, grp, 0);
    if (__all_sync(0xffffffffu, !in || grp == g0)) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long y = shfl_xor_u64(key, o);
            key = y > key ? y : key;
        }
        if ((threadIdx.x & 31) == 0 && g0 >= 0) atomicMax(b.group_key + g0, key);
    } else if (in) {
        atomicMax(b.group_key + grp, key);
    }
}

}  // namespace
}  // namespace grc
