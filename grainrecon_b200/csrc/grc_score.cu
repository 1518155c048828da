// grc_score.cu -- the (voxel, orientation) completeness scorer for sm_100a.
//
// One kernel scores trials = (voxel, orientation) pairs; the seeding scan
// (cuda_forward_comp), the grower (cuda_grow_indexed_region) and the
// candidate competition (cuda_forward_comp_compete) are work lists over it.
//
// Per trial the reference (forward_comp.m:18-82) walks every projection omega
// and every reflection hkl.  Here one CTA owns one trial at a time:
//   * per work item (one voxel, a run of its trials) the CTA builds an omega
//     table in shared memory: FP64 constants of the cone-beam geometry that do
//     not depend on the orientation, plus the FP32 incident direction rotated
//     back into the sample frame (k_w = Omega^T k_in);
//   * warps take omegas round-robin, lanes take reflections (up to 4 per lane,
//     the trial's G = S*U*B*h held in registers), and an FP32 prefilter
//     -(k_w . G) in (lambda_min |G|^2/4pi, lambda_max |G|^2/4pi), widened by a
//     margin far above its rounding error, drops the ~80% of reflections that
//     miss the energy window after 3 FMAs;
//   * survivors are compacted through a per-warp shared-memory queue and
//     evaluated 32 at a time with every lane busy: the exact FP64 window test,
//     the Bragg/cone-beam landing point and the tilted-detector intersection,
//     round-half-away pixel, detector and beam-stop tests;
//   * a selected reflection reads one rank code of the distance map; counts go
//     to warp registers, the code to a shared-memory histogram, from which the
//     exact median (MATLAB even-count rule) is read after the trial.  Medians
//     whose rank lies above the histogram are finished by refine_kernel with
//     10-bit radix passes.
#include <cuda_runtime.h>
#include <math_constants.h>
#include <stdint.h>

#include "grc_internal.h"
#include "grc_chain.cuh"

// Resident CTAs per SM the scoring kernel is compiled for (register budget).
#ifndef GRC_MIN_BLOCKS
#define GRC_MIN_BLOCKS 4
#endif
#ifndef GRC_SWEEP_BLOCKS
#define GRC_SWEEP_BLOCKS 3
#endif

namespace grc {
namespace {

// Counts + histogram of codes below kHistBins (scoring pass).
template <typename CodeT>
struct HistSink {
    const CodeT *codes;
    uint32_t *hist;
    uint32_t n_hit;
    int simu, inter, over;
    __device__ __forceinline__ void on(int64_t idx) {
        const bool ok = idx >= 0;
        uint32_t code = 0;
        if (ok) code = (uint32_t)__ldg(codes + idx);
        const bool inr = ok && code < (uint32_t)kHistBins;
        if (inr) atomicAdd(&hist[code], 1u);
        const unsigned mo = __ballot_sync(kFull, ok);
        const unsigned mh = __ballot_sync(kFull, ok && code < n_hit);
        const unsigned mi = __ballot_sync(kFull, inr);
        simu += __popc(mo);
        inter += __popc(mh);
        over += __popc(mo & ~mi);
    }
};

// One 10-bit radix digit pass for two target ranks (refine pass).
template <typename CodeT>
struct RadixSink {
    const CodeT *codes;
    uint32_t *ha, *hb;
    uint32_t pa, pb;
    int digit_shift, prefix_shift;
    uint32_t digit_mask;
    __device__ __forceinline__ void on(int64_t idx) {
        if (idx < 0) return;
        const uint32_t code = (uint32_t)__ldg(codes + idx);
        const uint32_t pre = prefix_shift >= 32 ? 0u : (code >> prefix_shift);
        const uint32_t d = (code >> digit_shift) & digit_mask;
        if (pre == pa) atomicAdd(&ha[d], 1u);
        if (pre == pb) atomicAdd(&hb[d], 1u);
    }
};

// Marks landing pixels (synthetic spot simulation).
struct MarkSink {
    uint8_t *mask;
    __device__ __forceinline__ void on(int64_t idx) {
        if (idx >= 0) mask[idx] = 1;
    }
};

// Per-trial context handed to run_trial.
struct TrialCtx {
    const RowF *rows;        // shared: omega table of the voxel
    const float4 *gw;        // shared: FP32 Gw table of the trial
    const float4 *win;       // shared: window thresholds per reflection (window_of)
    const double *sub;       // shared: FP64 S*U*B of the trial
    const double *vp;        // global: voxel position (FP64)
    const double2 *rot_cs;   // global
    const double *hkl;       // global
    const Geo *geo;          // global copy of the geometry (exact path)
    uint32_t *wq;            // shared: this warp's candidate queue (kQueueCap)
    uint32_t *fq;            // shared: this warp's ambiguous-item queue (kFallbackCap)
};

// Walk every (omega, reflection) of one trial; the sink sees each selected pixel.
template <int HPL, typename Sink>
__device__ __forceinline__ void run_trial(const Geo &g, const TrialCtx &tc, Sink &sink) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    float pfx[HPL], pfy[HPL], pfz[HPL], plo[HPL], phi[HPL];
#pragma unroll
    for (int j = 0; j < HPL; ++j) {
        const int ih = lane + 32 * j;
        if (ih < g.nhkl) {
            const float4 gv = tc.gw[ih];
            const float4 w = tc.win[ih];
            plo[j] = w.x;
            phi[j] = w.y;
            pfx[j] = gv.x;
            pfy[j] = gv.y;
            pfz[j] = gv.z;
        } else {
            plo[j] = CUDART_INF_F;
            phi[j] = -CUDART_INF_F;
            pfx[j] = pfy[j] = pfz[j] = 0.f;
        }
    }
    uint32_t *wq = tc.wq, *fq = tc.fq;
    int qn = 0, fn = 0;
    auto fast = [&](uint32_t item, bool valid) {
        const int iwi = (int)(item >> 8), ihi = (int)(item & 255u);
        int64_t r = -1;
        if (valid) {
            const float4 gv = tc.gw[ihi];
            const float4 w = tc.win[ihi];
            const int ip = landing_fp32(g, tc.rows[iwi], gv, w.z, w.w);
            r = ip >= 0 ? (int64_t)iwi * g.plane + ip : (int64_t)ip;
        }
        const bool amb = r == -2;
        const unsigned m = __ballot_sync(kFull, amb);
        if (amb) fq[fn + __popc(m & lt)] = item;
        fn += __popc(m);
        sink.on(r >= 0 ? r : -1);
    };
    auto exact = [&](uint32_t item, bool valid) {
        int64_t r = -1;
        if (valid) r = landing_exact(tc.geo, tc.rot_cs, tc.vp, tc.hkl, tc.sub, (int)(item >> 8), (int)(item & 255u));
        sink.on(r);
    };
    for (int iw = warp; iw < g.nrot; iw += kWarps) {
        const RowF &row = tc.rows[iw];
        const float kx = row.wx, ky = row.wy, kz = row.wz;
#pragma unroll
        for (int j = 0; j < HPL; ++j) {
            const float t = -fmaf(kx, pfx[j], fmaf(ky, pfy[j], kz * pfz[j]));
            const bool pass = (t > plo[j]) && (t < phi[j]);
            const unsigned m = __ballot_sync(kFull, pass);
            if (pass) wq[qn + __popc(m & lt)] = ((uint32_t)iw << 8) | (uint32_t)(lane + 32 * j);
            qn += __popc(m);
        }
        __syncwarp();
        while (qn >= 32) {
            qn -= 32;
            const uint32_t item = wq[qn + lane];
            __syncwarp();
            fast(item, true);
            __syncwarp();
            while (fn >= 32) {
                fn -= 32;
                const uint32_t it2 = fq[fn + lane];
                __syncwarp();
                exact(it2, true);
                __syncwarp();
            }
        }
    }
    if (qn > 0) {
        const bool valid = lane < qn;
        const uint32_t item = valid ? wq[lane] : 0u;
        __syncwarp();
        fast(item, valid);
        __syncwarp();
    }
    while (fn > 0) {
        const int take = fn < 32 ? fn : 32;
        fn -= take;
        const bool valid = lane < take;
        const uint32_t item = valid ? fq[fn + lane] : 0u;
        __syncwarp();
        exact(item, valid);
        __syncwarp();
    }
}

struct Smem {
    RowF *rows;
    float4 *gw;
    float4 *win;
    double *sub;
    uint32_t *h0, *h1;
    uint32_t *queue;
    uint32_t *fqueue;
};

__device__ __forceinline__ Smem carve(unsigned char *base, const Geo &g, int nhist) {
    Smem s;
    size_t off = 0;
    s.rows = (RowF *)(base + off);
    off = align16(off + sizeof(RowF) * g.nrot);
    s.gw = (float4 *)(base + off);
    off = align16(off + sizeof(float4) * g.nhkl);
    s.win = (float4 *)(base + off);
    off = align16(off + sizeof(float4) * g.nhkl);
    s.sub = (double *)(base + off);
    off = align16(off + sizeof(double) * 9);
    s.h0 = (uint32_t *)(base + off);
    off += sizeof(uint32_t) * kHistBins;
    s.h1 = nhist > 1 ? (uint32_t *)(base + off) : nullptr;
    off += nhist > 1 ? sizeof(uint32_t) * kHistBins : 0;
    s.queue = (uint32_t *)(base + off);
    off += sizeof(uint32_t) * kWarps * kQueueCap;
    s.fqueue = (uint32_t *)(base + off);
    return s;
}

__device__ __forceinline__ bool next_item(const Work &w, unsigned long long *counter, int64_t *s_item,
                                          int64_t &v, int64_t &t0, int64_t &t1) {
    if (threadIdx.x == 0) *s_item = (int64_t)atomicAdd(counter, 1ull);
    __syncthreads();
    const int64_t it = *s_item;
    __syncthreads();
    if (it >= w.n_items) return false;
    if (w.items) {
        const longlong4 e = w.items[it];
        v = e.x;
        t0 = e.y;
        t1 = e.z;
    } else {
        v = it / w.chunks_per_voxel;
        const int64_t c = it % w.chunks_per_voxel;
        t0 = v * w.n_or + c * w.chunk;
        const int64_t end = (v + 1) * w.n_or;
        t1 = t0 + w.chunk < end ? t0 + w.chunk : end;
    }
    return true;
}

__device__ __forceinline__ int64_t orient_of(const Work &w, int64_t t, int64_t v) {
    if (w.trial_orient) return (int64_t)w.trial_orient[t];
    return w.diag ? t : (t - v * w.n_or);
}

// Block-wide search of the smallest bins with cumulative count >= ra and >= rb.
__device__ void find_two_ranks(const uint32_t *hist, int ra, int rb, int *s_code, uint32_t *s_wsum) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    constexpr int per = kHistBins / kThreads;
    const int base = threadIdx.x * per;
    uint32_t c[per];
    uint32_t local = 0;
#pragma unroll
    for (int i = 0; i < per; ++i) {
        c[i] = hist[base + i];
        local += c[i];
    }
    uint32_t incl = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(kFull, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) s_wsum[warp] = incl;
    __syncthreads();
    uint32_t woff = 0;
    for (int i = 0; i < warp; ++i) woff += s_wsum[i];
    const uint32_t excl = incl - local + woff;
    const uint32_t r2[2] = {(uint32_t)ra, (uint32_t)rb};
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const uint32_t r = r2[q];
        if (excl < r && r <= excl + local) {
            uint32_t cum = excl;
#pragma unroll
            for (int i = 0; i < per; ++i) {
                cum += c[i];
                if (cum >= r) {
                    s_code[q] = base + i;
                    break;
                }
            }
        }
    }
}

template <int HPL, typename CodeT>
__global__ void __launch_bounds__(kThreads, GRC_MIN_BLOCKS) score_kernel(Geo g, ScoreBufs b, Work w) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const Smem sm = carve(smem_raw, g, 1);
    __shared__ int64_t s_item;
    __shared__ int s_simu, s_inter, s_over;
    __shared__ int s_code[2];
    __shared__ uint32_t s_wsum[kWarps];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint32_t *wq = sm.queue + warp * kQueueCap;
    uint32_t *fq = sm.fqueue + warp * kFallbackCap;
    const CodeT *codes = (const CodeT *)b.codes;
    unsigned long long *counter = (unsigned long long *)b.work_counter;
    int64_t v, t0, t1;
    while (next_item(w, counter, &s_item, v, t0, t1)) {
        if (t0 >= t1) continue;
        build_rows(g, b.rot_cs, b.vpos + 3 * v, sm.rows);
        const TrialCtx tc{sm.rows, sm.gw, sm.win, sm.sub, b.vpos + 3 * v, b.rot_cs, b.hkl, b.geo, wq, fq};
        for (int64_t t = t0; t < t1; ++t) {
            const int64_t o = orient_of(w, t, v);
            build_gw(g, b.hkl, b.U + 9 * o, sm.gw, sm.win, sm.sub);
            for (int i = threadIdx.x; i < kHistBins; i += kThreads) sm.h0[i] = 0;
            if (threadIdx.x == 0) {
                s_simu = s_inter = s_over = 0;
                s_code[0] = s_code[1] = -1;
            }
            __syncthreads();
            HistSink<CodeT> sink{codes, sm.h0, g.n_hit, 0, 0, 0};
            run_trial<HPL>(g, tc, sink);
            if (lane == 0) {
                atomicAdd(&s_simu, sink.simu);
                atomicAdd(&s_inter, sink.inter);
                atomicAdd(&s_over, sink.over);
            }
            __syncthreads();
            const int n = s_simu, inr = n - s_over;
            const int ra = (n + 1) / 2, rb = n / 2 + 1;
            const bool direct = n > 0 && rb <= inr;
            if (direct) find_two_ranks(sm.h0, ra, rb, s_code, s_wsum);
            __syncthreads();
            if (threadIdx.x == 0) {
                TrialRes r;
                r.simu = n;
                r.inter = s_inter;
                if (n == 0) {
                    r.median = 2000.0;  // forward_comp.m:89
                } else if (direct) {
                    const uint32_t ca = min((uint32_t)s_code[0], g.n_vals - 1u), cb = min((uint32_t)s_code[1], g.n_vals - 1u);
                    r.median = ((double)b.vals[ca] + (double)b.vals[cb]) / 2.0;
                } else {
                    r.median = CUDART_NAN;
                    atomicAdd(b.work_counter + 4, 1);
                }
                b.res[t] = r;
            }
        }
        __syncthreads();
    }
}

// Exact median for trials whose median rank lies beyond the histogram: radix
// select over the code bits, two ranks at once, one full trial walk per digit.
template <int HPL, typename CodeT>
__global__ void __launch_bounds__(kThreads, 2) refine_kernel(Geo g, ScoreBufs b, Work w) {
    if (b.work_counter[4] == 0) return;  // nothing to refine
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const Smem sm = carve(smem_raw, g, 2);
    __shared__ int64_t s_item;
    __shared__ int s_any;
    __shared__ uint32_t s_pa, s_pb, s_ra, s_rb;
    const int warp = threadIdx.x >> 5;
    uint32_t *wq = sm.queue + warp * kQueueCap;
    uint32_t *fq = sm.fqueue + warp * kFallbackCap;
    const CodeT *codes = (const CodeT *)b.codes;
    unsigned long long *counter = (unsigned long long *)(b.work_counter + 2);
    int64_t v, t0, t1;
    while (next_item(w, counter, &s_item, v, t0, t1)) {
        if (threadIdx.x == 0) s_any = 0;
        __syncthreads();
        for (int64_t t = t0 + threadIdx.x; t < t1; t += kThreads)
            if (isnan(b.res[t].median)) s_any = 1;
        __syncthreads();
        if (!s_any) continue;
        build_rows(g, b.rot_cs, b.vpos + 3 * v, sm.rows);
        __syncthreads();
        const TrialCtx tc{sm.rows, sm.gw, sm.win, sm.sub, b.vpos + 3 * v, b.rot_cs, b.hkl, b.geo, wq, fq};
        for (int64_t t = t0; t < t1; ++t) {
            if (!isnan(b.res[t].median)) continue;  // uniform: every thread reads the same value
            const int64_t o = orient_of(w, t, v);
            __syncthreads();
            build_gw(g, b.hkl, b.U + 9 * o, sm.gw, sm.win, sm.sub);
            const int n = b.res[t].simu;
            if (threadIdx.x == 0) {
                s_pa = s_pb = 0;
                s_ra = (uint32_t)((n + 1) / 2);
                s_rb = (uint32_t)(n / 2 + 1);
            }
            int pos = g.code_bits;
            while (pos > 0) {
                const int width = pos < 10 ? pos : 10;
                pos -= width;
                for (int i = threadIdx.x; i < kHistBins; i += kThreads) sm.h0[i] = sm.h1[i] = 0;
                __syncthreads();
                RadixSink<CodeT> sink{codes, sm.h0, sm.h1, s_pa, s_pb, pos, pos + width, (1u << width) - 1u};
                run_trial<HPL>(g, tc, sink);
                __syncthreads();
                if (threadIdx.x == 0) {
                    uint32_t cum = 0;
                    for (uint32_t d = 0; d < (1u << width); ++d) {
                        if (cum + sm.h0[d] >= s_ra) {
                            s_ra -= cum;
                            s_pa = (s_pa << width) | d;
                            break;
                        }
                        cum += sm.h0[d];
                    }
                    cum = 0;
                    for (uint32_t d = 0; d < (1u << width); ++d) {
                        if (cum + sm.h1[d] >= s_rb) {
                            s_rb -= cum;
                            s_pb = (s_pb << width) | d;
                            break;
                        }
                        cum += sm.h1[d];
                    }
                }
                __syncthreads();
            }
            if (threadIdx.x == 0) {
                const uint32_t ca = min(s_pa, g.n_vals - 1u), cb = min(s_pb, g.n_vals - 1u);
                b.res[t].median = ((double)b.vals[ca] + (double)b.vals[cb]) / 2.0;
            }
            __syncthreads();
        }
    }
}

// Synthetic spot simulation: every trial marks its selected landing pixels.
template <int HPL>
__global__ void __launch_bounds__(kThreads, 2) mark_kernel(Geo g, ScoreBufs b, Work w, uint8_t *mask) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const Smem sm = carve(smem_raw, g, 1);
    __shared__ int64_t s_item;
    const int warp = threadIdx.x >> 5;
    uint32_t *wq = sm.queue + warp * kQueueCap;
    uint32_t *fq = sm.fqueue + warp * kFallbackCap;
    unsigned long long *counter = (unsigned long long *)b.work_counter;
    int64_t v, t0, t1;
    while (next_item(w, counter, &s_item, v, t0, t1)) {
        if (t0 >= t1) continue;
        build_rows(g, b.rot_cs, b.vpos + 3 * v, sm.rows);
        const TrialCtx tc{sm.rows, sm.gw, sm.win, sm.sub, b.vpos + 3 * v, b.rot_cs, b.hkl, b.geo, wq, fq};
        for (int64_t t = t0; t < t1; ++t) {
            build_gw(g, b.hkl, b.U + 9 * orient_of(w, t, v), sm.gw, sm.win, sm.sub);
            __syncthreads();
            MarkSink sink{mask};
            run_trial<HPL>(g, tc, sink);
            __syncthreads();
        }
    }
}

// ---------------------------------------------------------------------------------
// Projection-window sweep.  One launch = one round: each CTA holds kSlots trials in
// shared memory (a 256-bin histogram of the 8-bit saturated codes, S*U*B) and every CTA
// walks the projections in windows of nwin at the same pace, so the map pixels being read
// belong to a few projections at a time and stay in L2.  The window is 32, 16 or 8
// projections: the widest whose omega rows keep the CTAs per SM of the 8-wide layout
// (fewer window barriers and row rebuilds per trial).
constexpr int kSlots = 96;      // most trials a CTA holds in one round
constexpr int kSlotsBulk = 64;  // tile of multi-round work and of explicit voxel lists
constexpr int kWinMin = 8;      // narrowest projection window
constexpr int kWinWide[2] = {32, 16};  // wider windows tried first (instantiated for these)
constexpr int kHist8Words = 128;  // 256 u16 bins per slot, two per word

__device__ __forceinline__ int64_t voxel_of(const Work &w, int64_t t) {
    if (w.trial_voxel) return (int64_t)w.trial_voxel[t];
    if (w.diag) return t;
    return t / w.n_or;
}

struct SweepSmem {
    RowF *rows;       // [rows_cap * nwin] rows of the current window, indexed vloc * nwin + wl
    float4 *hk;       // [nhkl] h as float
    uint32_t *hist;   // [slots * kHist8Words]; Nr_simu and Nr_intersect are read from it
    float *subf;      // [slots * 12]
    double *subd;     // [slots * 9]
    int *vloc;        // [slots]
    int64_t *vglob;   // [slots]
    int64_t *vlist;   // [slots]
    uint32_t *queue;  // [kWarps * kQueueCap]
    uint32_t *fqueue; // [kWarps * kFallbackCap]
};

// Shared-memory layout of one CTA holding `slots` trials and rows of `rows_cap` voxels:
// kSweepParts arrays, offsets returned in offs[].
constexpr int kSweepParts = 10;
__host__ __device__ inline size_t sweep_smem_layout(int nhkl, int rows_cap, int slots, int nwin, size_t *offs,
                                                    int mode = kScanFull) {
    size_t o = 0, i = 0;
    auto put = [&](size_t bytes) {
        o = (o + 15) & ~size_t(15);
        offs[i++] = o;
        o += bytes;
    };
    put(sizeof(RowF) * rows_cap * nwin);
    put(sizeof(float4) * nhkl);
    put(sizeof(uint32_t) * slots * (mode == kScanFull ? kHist8Words : 1));
    put(sizeof(float) * slots * 12);
    put(sizeof(double) * slots * 9);
    put(sizeof(int) * slots);
    put(sizeof(int64_t) * slots);
    put(sizeof(int64_t) * slots);
    put(sizeof(uint32_t) * kWarps * kQueueCap);
    put(sizeof(uint32_t) * kWarps * kFallbackCap);
    return (o + 15) & ~size_t(15);
}

__device__ __forceinline__ SweepSmem sweep_carve(unsigned char *base, int nhkl, int rows_cap, int slots, int nwin,
                                                 int mode) {
    size_t offs[kSweepParts];
    sweep_smem_layout(nhkl, rows_cap, slots, nwin, offs, mode);
    SweepSmem m;
    m.rows = (RowF *)(base + offs[0]);
    m.hk = (float4 *)(base + offs[1]);
    m.hist = (uint32_t *)(base + offs[2]);
    m.subf = (float *)(base + offs[3]);
    m.subd = (double *)(base + offs[4]);
    m.vloc = (int *)(base + offs[5]);
    m.vglob = (int64_t *)(base + offs[6]);
    m.vlist = (int64_t *)(base + offs[7]);
    m.queue = (uint32_t *)(base + offs[8]);
    m.fqueue = (uint32_t *)(base + offs[9]);
    return m;
}

// MODE kScanFull: per slot a 256-bin histogram of the 8-bit codes (counts and exact median);
// kScanComp: per slot one packed counter (Nr_simu in the low 16 bits, Nr_intersect in the high
// 16; both stay below 2^16 because the sweep takes at most 65,535 reflections per trial), the hit
// read from the bit-packed mask, no median.
template <int HPL, int WIN, int MODE>
__global__ void __launch_bounds__(kThreads, GRC_SWEEP_BLOCKS) sweep_kernel(Geo g, ScoreBufs b, Work w, int64_t round_base,
                                                            int64_t n_trials, int rows_cap, int slots) {
    constexpr int nwin = WIN;  // projections per window
    const int64_t cta_base = round_base + (int64_t)blockIdx.x * slots;
    if (cta_base >= n_trials) return;
    const int nslot = (int)min((int64_t)slots, n_trials - cta_base);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const SweepSmem sm = sweep_carve(smem_raw, g.nhkl, rows_cap, slots, nwin, MODE);
    __shared__ int s_nv, s_next;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const unsigned lt = (1u << lane) - 1u;
    uint32_t *wq = sm.queue + warp * kQueueCap;
    uint32_t *fq = sm.fqueue + warp * kFallbackCap;

    // ---- set-up: per-slot S*U*B, voxels, zeroed counters and histograms
    if (tid < nslot) {
        const int64_t t = cta_base + tid;
        const int64_t v = voxel_of(w, t);
        const int64_t o = orient_of(w, t, v);
        double SUB[9];
        sub_matrix(g, b.U + 9 * o, SUB);
#pragma unroll
        for (int i = 0; i < 9; ++i) {
            sm.subd[9 * tid + i] = SUB[i];
            sm.subf[12 * tid + i] = (float)SUB[i];
        }
        sm.vglob[tid] = v;
    }
    for (int i = tid; i < slots * (MODE == kScanFull ? kHist8Words : 1); i += kThreads) sm.hist[i] = 0;
    for (int i = tid; i < g.nhkl; i += kThreads)
        sm.hk[i] = make_float4((float)b.hkl[3 * i], (float)b.hkl[3 * i + 1], (float)b.hkl[3 * i + 2], 0.f);
    __syncthreads();
    if (tid == 0) {
        int nv = 0;
        for (int s = 0; s < nslot; ++s) {
            if (s == 0 || sm.vglob[s] != sm.vglob[s - 1]) sm.vlist[nv++] = sm.vglob[s];
            sm.vloc[s] = nv - 1;
        }
        s_nv = nv;
    }
    __syncthreads();
    const int nv = s_nv;
    const int64_t pw = b.plane_words;

    // Selected pixels reach the histogram one batch late: the code of batch k is loaded
    // when batch k is evaluated and applied after batch k+1 has been computed, so the
    // L2 latency of the gather overlaps the next landing computations.  The histogram is
    // the only per-selection update: Nr_simu is its total and Nr_intersect the total of its
    // codes below n_hit (< 255, so the saturated bin never holds a hit).
    int pend_off = -1;   // full: the pending offset in the projection window; completeness: its bit (or -1)
    int pend_slot = 0;
    uint32_t pend_code = 0;  // full: the 8-bit code; completeness: the mask word
    auto apply_pending = [&]() {
        if (pend_off >= 0) {
            if (MODE == kScanFull)
                atomicAdd(&sm.hist[pend_slot * kHist8Words + (pend_code >> 1)], 1u << ((pend_code & 1u) * 16));
            else
                atomicAdd(&sm.hist[pend_slot], 1u + (((pend_code >> pend_off) & 1u) << 16));
        }
        pend_off = -1;
    };

    for (int w0 = 0; w0 < g.nrot; w0 += nwin) {
        const int nw = min(nwin, g.nrot - w0);
        // codes of the window's first pixel; offsets within the window fit 32 bits
        // (nwin * plane < 2^31, launch_sweep_t)
        const uint8_t *wcodes = MODE == kScanFull ? b.codes8 + (int64_t)w0 * g.plane : nullptr;
        const uint32_t *wbits = MODE == kScanComp ? b.bits + (int64_t)w0 * pw : nullptr;
        // warp-synchronous: every lane calls it once per batch; ip = in-plane pixel or -1
        auto sink = [&](int wl, int ip, int s) {
            uint32_t code = 0;
            int off = -1;
            if (ip >= 0) {
                if (MODE == kScanFull) {
                    off = wl * (int)g.plane + ip;
                    code = __ldg(wcodes + off);
                } else {
                    off = ip & 31;
                    code = __ldg(wbits + (int64_t)wl * pw + (ip >> 5));
                }
            }
            apply_pending();
            pend_off = off;
            pend_slot = s;
            pend_code = code;
        };
        // ---- omega rows of this window for every voxel of the round
        for (int i = tid; i < nv * nw; i += kThreads) {
            const int vl = i / nw, wl = i - vl * nw;
            sm.rows[vl * nwin + wl] = row_f32(g, omega_row(g, b.rot_cs[w0 + wl], b.vpos + 3 * sm.vlist[vl]));
        }
        if (tid == 0) s_next = 0;
        __syncthreads();
        int qn = 0, fn = 0;
        auto fast = [&](uint32_t item, bool valid) {
            int ip = -1;
            const int s = (int)(item >> 16), wl = (int)((item >> 8) & 255u), ih = (int)(item & 255u);
            if (valid) {
                const float4 gv = gw_of(sm.subf + 12 * s, sm.hk[ih]);
                const float4 win = window_f(g, gv);
                ip = landing_fp32(g, sm.rows[sm.vloc[s] * nwin + wl], gv, win.z, win.w);
#ifdef GRC_AUDIT
                const int r = ip >= 0 ? wl * (int)g.plane + ip : ip;
                // audit build: every certain FP32 decision is re-decided by the FP64 path
                if (r != -2) {
                    const int64_t r64 = landing_exact(b.geo, b.rot_cs, b.vpos + 3 * sm.vglob[s], b.hkl,
                                                      sm.subd + 9 * s, w0 + wl, ih);
                    atomicAdd((unsigned long long *)(b.work_counter + 6), 1ull);
                    if ((r64 >= 0 ? (int)(r64 - (int64_t)w0 * g.plane) : -1) != r) atomicAdd(b.work_counter + 5, 1);
                }
#endif
            }
            const bool amb = ip == -2;
            const unsigned m = __ballot_sync(kFull, amb);
            if (amb) fq[fn + __popc(m & lt)] = item;
            fn += __popc(m);
            sink(wl, ip >= 0 ? ip : -1, s);
        };
        auto exact = [&](uint32_t item, bool valid) {
            const int s = (int)(item >> 16), wl = (int)((item >> 8) & 255u), ih = (int)(item & 255u);
            int ip = -1;
            if (valid) {
                const int64_t r64 =
                    landing_exact(b.geo, b.rot_cs, b.vpos + 3 * sm.vglob[s], b.hkl, sm.subd + 9 * s, w0 + wl, ih);
                ip = r64 >= 0 ? (int)(r64 - (int64_t)(w0 + wl) * g.plane) : -1;
            }
            sink(wl, ip, s);
        };
        auto drain = [&](bool all) {
            while (qn >= 32 || (all && qn > 0)) {
                const int take = qn >= 32 ? 32 : qn;
                qn -= take;
                const bool valid = lane < take;
                const uint32_t item = valid ? wq[qn + lane] : 0u;
                __syncwarp();
                fast(item, valid);
                __syncwarp();
                while (fn >= 32) {
                    fn -= 32;
                    const uint32_t it2 = fq[fn + lane];
                    __syncwarp();
                    exact(it2, true);
                    __syncwarp();
                }
            }
            if (all) {
                while (fn > 0) {
                    const int tk = fn >= 32 ? 32 : fn;
                    fn -= tk;
                    const bool v2 = lane < tk;
                    const uint32_t it2 = v2 ? fq[fn + lane] : 0u;
                    __syncwarp();
                    exact(it2, v2);
                    __syncwarp();
                }
            }
        };
        // slots are handed out one at a time, so the warps of a CTA reach the end-of-window
        // barrier together however unevenly the selected reflections fall on the slots
        for (;;) {
            int s = 0;
            if (lane == 0) s = atomicAdd(&s_next, 1);
            s = __shfl_sync(kFull, s, 0);
            if (s >= nslot) break;
            const float *sf = sm.subf + 12 * s;
            float gx[HPL], gy[HPL], gz[HPL], lo[HPL], hi[HPL];
#pragma unroll
            for (int j = 0; j < HPL; ++j) {
                // h re-read from shared memory at each slot: holding it in registers for the
                // whole kernel costs spills of the 80-register budget
                const int ihj = lane + 32 * j;
                const float4 gv = gw_of(sf, ihj < g.nhkl ? sm.hk[ihj] : make_float4(0.f, 0.f, 0.f, 0.f));
                const float4 win = window_f(g, gv);
                const bool real = lane + 32 * j < g.nhkl;
                gx[j] = gv.x;
                gy[j] = gv.y;
                gz[j] = gv.z;
                lo[j] = real ? win.x : CUDART_INF_F;
                hi[j] = real ? win.y : -CUDART_INF_F;
            }
            const RowF *vr = sm.rows + sm.vloc[s] * nwin;
            for (int wl = 0; wl < nw; ++wl) {
                const float4 kwv = reinterpret_cast<const float4 *>(vr + wl)[3];
                const float kx = kwv.x, ky = kwv.y, kz = kwv.z;
#pragma unroll
                for (int j = 0; j < HPL; ++j) {
                    const float t = -fmaf(kx, gx[j], fmaf(ky, gy[j], kz * gz[j]));
                    const bool pass = (t > lo[j]) && (t < hi[j]);
                    const unsigned m = __ballot_sync(kFull, pass);
                    if (pass)
                        wq[qn + __popc(m & lt)] =
                            ((uint32_t)s << 16) | ((uint32_t)wl << 8) | (uint32_t)(lane + 32 * j);
                    qn += __popc(m);
                }
                __syncwarp();
                drain(false);
            }
        }
        drain(true);
        apply_pending();
        __syncthreads();  // rows are rebuilt for the next window
    }

    // ---- finalize: one warp per slot, exact median from the 8-bit histogram; or the counters
    if constexpr (MODE == kScanFull) {
        for (int s = warp; s < nslot; s += kWarps) hist8_finish(g, b, sm.hist + s * kHist8Words, cta_base + s);
    } else {
        for (int base = warp * 32; base < nslot; base += kWarps * 32) {
            const int s = base + lane;
            const bool in = s < nslot;
            int simu = 0, inter = 0;
            if (in) {
                const uint32_t c = sm.hist[s];
                simu = (int)(c & 0xffffu);
                inter = (int)(c >> 16);
                TrialRes r;
                r.simu = simu;
                r.inter = inter;
                r.median = CUDART_NAN;  // not computed in this mode
                b.res[cta_base + s] = r;
            }
            if (b.group_key) fold_group_key(b, in, cta_base + s, simu, inter);
        }
    }
}

// Exact median for the trials listed by the sweep: full omega table, full-width codes,
// 10-bit radix passes (random gathers; these trials are rare).
template <int HPL, typename CodeT>
__global__ void __launch_bounds__(kThreads, 2) refine_list_kernel(Geo g, ScoreBufs b, Work w) {
    const int n_list = b.work_counter[4];
    if (n_list == 0) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const Smem sm = carve(smem_raw, g, 2);
    __shared__ uint32_t s_pa, s_pb, s_ra, s_rb;
    const int warp = threadIdx.x >> 5;
    uint32_t *wq = sm.queue + warp * kQueueCap;
    uint32_t *fq = sm.fqueue + warp * kFallbackCap;
    const CodeT *codes = (const CodeT *)b.codes;
    for (int k = blockIdx.x; k < n_list; k += gridDim.x) {
        const int64_t t = b.refine_list[k];
        const int64_t v = voxel_of(w, t);
        const int64_t o = orient_of(w, t, v);
        __syncthreads();
        build_rows(g, b.rot_cs, b.vpos + 3 * v, sm.rows);
        build_gw(g, b.hkl, b.U + 9 * o, sm.gw, sm.win, sm.sub);
        const TrialCtx tc{sm.rows, sm.gw, sm.win, sm.sub, b.vpos + 3 * v, b.rot_cs, b.hkl, b.geo, wq, fq};
        const int n = b.res[t].simu;
        if (threadIdx.x == 0) {
            s_pa = s_pb = 0;
            s_ra = (uint32_t)((n + 1) / 2);
            s_rb = (uint32_t)(n / 2 + 1);
        }
        int pos = g.code_bits;
        while (pos > 0) {
            const int width = pos < 10 ? pos : 10;
            pos -= width;
            for (int i = threadIdx.x; i < kHistBins; i += kThreads) sm.h0[i] = sm.h1[i] = 0;
            __syncthreads();
            RadixSink<CodeT> sink{codes, sm.h0, sm.h1, s_pa, s_pb, pos, pos + width, (1u << width) - 1u};
            run_trial<HPL>(g, tc, sink);
            __syncthreads();
            if (threadIdx.x == 0) {
                uint32_t cum = 0;
                for (uint32_t d = 0; d < (1u << width); ++d) {
                    if (cum + sm.h0[d] >= s_ra) {
                        s_ra -= cum;
                        s_pa = (s_pa << width) | d;
                        break;
                    }
                    cum += sm.h0[d];
                }
                cum = 0;
                for (uint32_t d = 0; d < (1u << width); ++d) {
                    if (cum + sm.h1[d] >= s_rb) {
                        s_rb -= cum;
                        s_pb = (s_pb << width) | d;
                        break;
                    }
                    cum += sm.h1[d];
                }
            }
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            const uint32_t ca = min(s_pa, g.n_vals - 1u), cb = min(s_pb, g.n_vals - 1u);
            b.res[t].median = ((double)b.vals[ca] + (double)b.vals[cb]) / 2.0;
        }
    }
}

template <typename K>
cudaError_t prep_launch(K kern, size_t smem, int num_sms, int64_t n_items, int *grid_out) {
    int per_sm = 0;
    const cudaError_t e = occupancy_for((const void *)kern, smem, &per_sm);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    int64_t grid = (int64_t)per_sm * num_sms;
    if (grid > n_items) grid = n_items;
    if (grid < 1) grid = 1;
    *grid_out = (int)grid;
    return cudaSuccess;
}

template <int HPL, typename CodeT>
cudaError_t launch_score_t(const Geo &g, const ScoreBufs &b, const Work &w, int num_sms, cudaStream_t s,
                           cudaEvent_t ev0, cudaEvent_t ev1, int *launches) {
    const size_t smem = score_smem_bytes(g.nrot, g.nhkl);
    const size_t smem_r = refine_smem_bytes(g.nrot, g.nhkl);
    int grid = 0, grid_r = 0;
    cudaError_t e = prep_launch(score_kernel<HPL, CodeT>, smem, num_sms, w.n_items, &grid);
    if (e != cudaSuccess) return e;
    e = prep_launch(refine_kernel<HPL, CodeT>, smem_r, num_sms, w.n_items, &grid_r);
    if (e != cudaSuccess) return e;
    // counters: [0..1] main work (u64), [2..3] refine work (u64), [4] refine needed
    e = cudaMemsetAsync(b.work_counter, 0, 8 * sizeof(int), s);
    if (e != cudaSuccess) return e;
    if (ev0) cudaEventRecord(ev0, s);
    score_kernel<HPL, CodeT><<<grid, kThreads, smem, s>>>(g, b, w);
    if (ev1) cudaEventRecord(ev1, s);
    refine_kernel<HPL, CodeT><<<grid_r, kThreads, smem_r, s>>>(g, b, w);
    *launches += 2;
    return cudaGetLastError();
}


template <int HPL, typename CodeT, int MODE>
cudaError_t launch_sweep_t(const Geo &g, const ScoreBufs &b, const Work &w, int64_t n_trials, int num_sms,
                           cudaStream_t s, cudaEvent_t ev0, cudaEvent_t ev1, int *launches, int max_slots) {
    // The tile is kSlotsBulk trials per CTA.  An implicit seeding list (a few voxels per CTA) may
    // take up to kSlots when that fits the whole call into one round -- a one-seed scan of 32,768
    // orientations then runs as one round of 74 trials per CTA instead of two of 37.  Explicit
    // voxel lists keep one row set per trial in shared memory and stay at kSlotsBulk unless the
    // caller asks for another tile.  Shared memory is sized by the tile actually used.
    const bool explicit_voxels = w.trial_voxel || w.diag || w.n_or <= 0;
    const bool caller_tile = max_slots >= 1 && max_slots <= kSlots;
    if (!caller_tile) max_slots = kSlotsBulk;
    auto rows_for = [&](int sl) {  // distinct voxels one CTA can meet among sl consecutive trials
        int rc = (int)(w.n_or >= sl ? 2 : (w.n_or > 0 ? sl / w.n_or + 2 : sl));
        if (explicit_voxels) {
            // sl consecutive trials overlap at most ceil(sl/32) + 1 aligned blocks of 32, each with
            // at most starts_per_32 run starts: a seed-major list needs a few row sets, not sl
            rc = w.starts_per_32 > 0 ? 1 + ((sl + 31) / 32 + 1) * w.starts_per_32 : sl;
        }
        return rc > sl ? sl : rc;
    };
    size_t offs[kSweepParts];
    const size_t smem_max = sweep_smem_layout(g.nhkl, rows_for(max_slots), max_slots, kWinMin, offs, MODE);
    const size_t smem_r = refine_smem_bytes(g.nrot, g.nhkl);
    int per_sm = 0;
    using SweepFn = void (*)(Geo, ScoreBufs, Work, int64_t, int64_t, int, int);
    const SweepFn k8 = sweep_kernel<HPL, kWinMin, MODE>;
    cudaError_t e = occupancy_for((const void *)k8, smem_max, &per_sm);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    int grid_r = 0;
    e = prep_launch(refine_list_kernel<HPL, CodeT>, smem_r, num_sms, (int64_t)num_sms * 4, &grid_r);
    if (e != cudaSuccess) return e;
    const int64_t grid = (int64_t)per_sm * num_sms;
    if (!caller_tile && !explicit_voxels && n_trials > grid * max_slots && n_trials <= grid * kSlots) {
        // one round of up to kSlots trials per CTA, if the larger tile keeps the same CTAs per SM
        int per_sm1 = 0;
        const size_t smem1 = sweep_smem_layout(g.nhkl, rows_for(kSlots), kSlots, kWinMin, offs, MODE);
        if (occupancy_for((const void *)k8, smem1, &per_sm1) == cudaSuccess && per_sm1 == per_sm) {
            max_slots = kSlots;
        }
    }
    // rounds of equal size: slots per CTA chosen so the last round is not a sliver
    const int64_t rounds = (n_trials + grid * max_slots - 1) / (grid * max_slots);
    int slots = (int)((n_trials + rounds * grid - 1) / (rounds * grid));
    if (slots < 1) slots = 1;
    const int rows_cap = rows_for(slots);
    // the widest projection window whose rows keep the grid's CTAs per SM (and 32-bit map
    // offsets within a window)
    SweepFn kern = k8;
    size_t smem = sweep_smem_layout(g.nhkl, rows_cap, slots, kWinMin, offs, MODE);
    bool refused = false;
    for (int cand : kWinWide) {
        if ((int64_t)cand * g.plane > 2147483647LL) continue;
        const SweepFn kc = cand == 32 ? (SweepFn)sweep_kernel<HPL, 32, MODE> : (SweepFn)sweep_kernel<HPL, 16, MODE>;
        const size_t smem_c = sweep_smem_layout(g.nhkl, rows_cap, slots, cand, offs, MODE);
        int per_c = 0;
        if (occupancy_for((const void *)kc, smem_c, &per_c) != cudaSuccess) {
            refused = true;  // more shared memory than a CTA may have: not this window
            continue;
        }
        if (per_c >= per_sm) {
            kern = kc;
            smem = smem_c;
            break;
        }
    }
    if (refused) cudaGetLastError();  // the refused query is not an error of this launch
    e = allow_smem((const void *)kern, smem);
    if (e != cudaSuccess) return e;
    const int64_t per_round = grid * slots;
    e = cudaMemsetAsync(b.work_counter, 0, 8 * sizeof(int), s);
    if (e != cudaSuccess) return e;
    if (ev0) cudaEventRecord(ev0, s);
    for (int64_t base = 0; base < n_trials; base += per_round) {
        const int64_t left = (n_trials - base + slots - 1) / slots;
        const int gr = (int)(left < grid ? left : grid);
        kern<<<gr, kThreads, smem, s>>>(g, b, w, base, n_trials, rows_cap, slots);
        ++*launches;
    }
    if (ev1) cudaEventRecord(ev1, s);
    if (MODE == kScanFull) {  // completeness mode has no median to refine
        refine_list_kernel<HPL, CodeT><<<grid_r, kThreads, smem_r, s>>>(g, b, w);
        ++*launches;
    }
    return cudaGetLastError();
}

template <int HPL>
cudaError_t launch_mark_t(const Geo &g, const ScoreBufs &b, const Work &w, int num_sms, uint8_t *mask,
                          cudaStream_t s) {
    const size_t smem = score_smem_bytes(g.nrot, g.nhkl);
    int grid = 0;
    cudaError_t e = prep_launch(mark_kernel<HPL>, smem, num_sms, w.n_items, &grid);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(b.work_counter, 0, 8 * sizeof(int), s);
    if (e != cudaSuccess) return e;
    mark_kernel<HPL><<<grid, kThreads, smem, s>>>(g, b, w, mask);
    return cudaGetLastError();
}


// ---- spot pairing (forward_comp_pair_spots.m:60-85) ------------------------------------------
// For every selected reflection of a trial whose pixel is a hit, the nearest measured spot
// centroid of that projection (first in list order among equal distances) is paired when it
// lies closer than min(sqrt(area), 15) pixels.  The spot index holds, per projection, the spots
// of each cell of cell_px x cell_px pixels in list order.
// One selected (projection, reflection) item of a trial: the FP64 landing, the hit test and the
// nearest centroid.
template <typename CodeT>
__device__ __forceinline__ void pair_item(const Geo &g, const ScoreBufs &b, const SpotIndex &si, int64_t t,
                                          const OmegaRow &r, const double4 gv, int iw, int ih, PairRec *out,
                                          int64_t cap, unsigned long long *count) {
    const CodeT *codes = (const CodeT *)b.codes;
    double lam = 0.0;
    const int64_t idx = landing_fp64(g, r, gv.x, gv.y, gv.z, iw, &lam);
    if (idx < 0) return;
    const uint32_t code = (uint32_t)codes[idx];
    const int64_t in_plane = idx - (int64_t)iw * g.plane;
    const int dety = (int)(in_plane / g.detzsize) + 1, detz = (int)(in_plane % g.detzsize) + 1;
    const int cy0 = max(0, (dety - 16) / si.cell_px), cy1 = min(si.ncy - 1, (dety + 14) / si.cell_px);
    const int cz0 = max(0, (detz - 16) / si.cell_px), cz1 = min(si.ncz - 1, (detz + 14) / si.cell_px);
    // cells cz0..cz1 of one cell row are consecutive in the index, so a row's spots are one range
    // of cell_ids; the first row's bounds are read before the hit test, beside the code
    const int64_t row0 = ((int64_t)iw * si.ncy + cy0) * si.ncz;
    int64_t q0 = si.cell_off[row0 + cz0], q1 = si.cell_off[row0 + cz1 + 1];
    if (code >= g.n_hit) return;
    int best = -1;
    double bd = 0.0;
    for (int cy = cy0; cy <= cy1; ++cy) {
        if (cy > cy0) {
            const int64_t row = ((int64_t)iw * si.ncy + cy) * si.ncz;
            q0 = si.cell_off[row + cz0];
            q1 = si.cell_off[row + cz1 + 1];
        }
        for (int64_t q = q0; q < q1; ++q) {
            const int id = si.cell_ids[q];
            const double dy = __dsub_rn(si.yza[3 * id], (double)dety);
            const double dz = __dsub_rn(si.yza[3 * id + 1], (double)detz);
            const double d = sqrt(__dadd_rn(__dmul_rn(dy, dy), __dmul_rn(dz, dz)));
            if (best < 0 || d < bd || (d == bd && id < best)) {
                best = id;
                bd = d;
            }
        }
    }
    if (best < 0 || !(bd < fmin(sqrt(si.yza[3 * best + 2]), 15.0))) return;
    const unsigned long long slot = atomicAdd(count, 1ull);
    if ((int64_t)slot < cap) {
        PairRec p;
        p.trial = (int32_t)t;
        p.iw = iw;
        p.ih = ih;
        p.spot = best;
        p.dety = dety;
        p.detz = detz;
        p.exp_y = si.yza[3 * best];
        p.exp_z = si.yza[3 * best + 1];
        p.area = si.yza[3 * best + 2];
        p.energy_kev = 12.398 / lam;
        p.dis = (double)b.vals[min(code, g.n_vals - 1u)];
        out[slot] = p;
    }
}

constexpr int kPairThreads = 128, kPairWarps = kPairThreads / 32, kPairQueue = 64;

__host__ __device__ inline size_t pair_smem_bytes(int nrot, int nhkl) {
    return sizeof(double4) * nhkl + sizeof(double) * 10 + sizeof(OmegaRow) * nrot +
           sizeof(uint32_t) * kPairWarps * kPairQueue;
}

// One CTA per trial (grid-stride).  The trial's omega rows and G vectors (S*U*B*h with |G|) go to
// shared memory; each warp tests 32 (projection, reflection) pairs at a time against a window
// slightly wider than the landing's own (a superset: landing_fp64 makes the decision), queues
// the passing items and runs the FP64 landing and the centroid search on full batches of 32.
template <typename CodeT>
__global__ void __launch_bounds__(kPairThreads) pair_kernel(Geo g, ScoreBufs b, int64_t n, SpotIndex si,
                                                            PairRec *out, int64_t cap,
                                                            unsigned long long *count) {
    extern __shared__ __align__(16) unsigned char pair_smem[];
    double4 *gws = (double4 *)pair_smem;
    double *sub = (double *)(gws + g.nhkl);
    OmegaRow *rows = (OmegaRow *)(sub + 10);
    uint32_t *queue = (uint32_t *)(rows + g.nrot);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const unsigned lt = (1u << lane) - 1u;
    uint32_t *wq = queue + warp * kPairQueue;
    const int nh = g.nhkl, P = g.nrot * g.nhkl;
    for (int64_t t = blockIdx.x; t < n; t += gridDim.x) {
        __syncthreads();  // the previous trial's tables are no longer read
        if (tid == 0) sub_matrix(g, b.U + 9 * t, sub);
        const double *vp = b.vpos + 3 * t;
        for (int iw = tid; iw < g.nrot; iw += kPairThreads) rows[iw] = omega_row(g, b.rot_cs[iw], vp);
        __syncthreads();
        for (int ih = tid; ih < nh; ih += kPairThreads) {
            const double h = b.hkl[3 * ih], k = b.hkl[3 * ih + 1], l = b.hkl[3 * ih + 2];
            const double x = sub[0] * h + sub[1] * k + sub[2] * l;
            const double y = sub[3] * h + sub[4] * k + sub[5] * l;
            const double z = sub[6] * h + sub[7] * k + sub[8] * l;
            gws[ih] = make_double4(x, y, z, sqrt(x * x + y * y + z * z));
        }
        __syncthreads();
        int qn = 0;
        auto drain = [&](int take) {
            const bool valid = lane < take;
            const uint32_t it = valid ? wq[qn + lane] : 0u;
            __syncwarp();
            if (valid) {
                const int iw = (int)(it >> 8), ih = (int)(it & 255u);
                pair_item<CodeT>(g, b, si, t, rows[iw], gws[ih], iw, ih, out, cap, count);
            }
            __syncwarp();
        };
        for (int base = warp * 32; base < P; base += kPairThreads) {
            const int p = base + lane;
            bool pass = false;
            uint32_t item = 0;
            if (p < P) {
                const int iw = p / nh, ih = p - iw * nh;
                const OmegaRow &r = rows[iw];
                const double4 gv = gws[ih];
                // cos(beta) and 2 d sin(theta) as landing_fp64 forms them, tested with a margin
                const double Gtx = r.c * gv.x - r.s * gv.y, Gty = r.s * gv.x + r.c * gv.y;
                const double x = (r.kx * Gtx + r.ky * Gty + r.kz * gv.z) / gv.w;
                const double lam = 2.0 * (2.0 * CUDART_PI / gv.w) * (-x);
                pass = x < 1e-9 && x > g.cbmax - 1e-9 && lam > g.lmin * (1.0 - 1e-9) &&
                       lam < g.lmax * (1.0 + 1e-9);
                item = ((uint32_t)iw << 8) | (uint32_t)ih;
            }
            const unsigned bm = __ballot_sync(kFull, pass);
            if (pass) wq[qn + __popc(bm & lt)] = item;
            qn += __popc(bm);
            __syncwarp();
            if (qn >= 32) {
                qn -= 32;
                drain(32);
            }
        }
        if (qn > 0) {
            const int take = qn;
            qn = 0;
            drain(take);
        }
    }
}
}  // namespace

size_t score_smem_bytes(int nrot, int nhkl) {
    size_t off = 0;
    off = (off + sizeof(RowF) * nrot + 15) & ~size_t(15);
    off = (off + sizeof(float4) * nhkl + 15) & ~size_t(15);
    off = (off + sizeof(float4) * nhkl + 15) & ~size_t(15);
    off = (off + sizeof(double) * 9 + 15) & ~size_t(15);
    off += sizeof(uint32_t) * kHistBins;
    off += sizeof(uint32_t) * kWarps * (kQueueCap + kFallbackCap);
    return off;
}

size_t refine_smem_bytes(int nrot, int nhkl) { return score_smem_bytes(nrot, nhkl) + sizeof(uint32_t) * kHistBins; }

cudaError_t launch_score(const Geo &g, const ScoreBufs &b, const Work &w, int num_sms, cudaStream_t s,
                         cudaEvent_t ev0, cudaEvent_t ev1, int *launches) {
    const int hpl = (g.nhkl + 31) / 32;
    const bool c16 = g.code_bits <= 16;
#define GRC_DISPATCH(H)                                                                        \
    if (hpl == H)                                                                              \
        return c16 ? launch_score_t<H, uint16_t>(g, b, w, num_sms, s, ev0, ev1, launches)     \
                   : launch_score_t<H, uint32_t>(g, b, w, num_sms, s, ev0, ev1, launches);
    GRC_DISPATCH(1)
    GRC_DISPATCH(2)
    GRC_DISPATCH(3)
    GRC_DISPATCH(4)
#undef GRC_DISPATCH
    return cudaErrorInvalidValue;
}

cudaError_t launch_simulate_work(const Geo &g, const ScoreBufs &b, const Work &w, int num_sms, uint8_t *mask,
                                 cudaStream_t s) {
    const int hpl = (g.nhkl + 31) / 32;
    switch (hpl) {
        case 1: return launch_mark_t<1>(g, b, w, num_sms, mask, s);
        case 2: return launch_mark_t<2>(g, b, w, num_sms, mask, s);
        case 3: return launch_mark_t<3>(g, b, w, num_sms, mask, s);
        case 4: return launch_mark_t<4>(g, b, w, num_sms, mask, s);
        default: return cudaErrorInvalidValue;
    }
}

int64_t sweep_round_trials(const Geo &g, int num_sms) {
    // 16-bit per-slot counters and histogram bins; hit codes must stay below the saturation code
    // 32-bit offsets within a projection window
    if (g.n_hit >= 255u || g.nhkl > 128 || (int64_t)g.nrot * g.nhkl > 65535 ||
        (int64_t)kWinMin * g.plane > 2147483647LL)
        return 0;
    return (int64_t)num_sms * GRC_SWEEP_BLOCKS * kSlotsBulk;
}

cudaError_t launch_sweep(const Geo &g, const ScoreBufs &b, const Work &w, int64_t n_trials, int num_sms,
                         cudaStream_t s, cudaEvent_t ev0, cudaEvent_t ev1, int *launches, int max_slots, int mode) {
    const int hpl = (g.nhkl + 31) / 32;
    const bool c16 = g.code_bits <= 16;
    if (mode == kScanComp && !b.bits) return cudaErrorInvalidValue;
#define GRC_DISPATCH(H)                                                                                          \
    if (hpl == H) {                                                                                              \
        if (mode == kScanComp)                                                                                   \
            return launch_sweep_t<H, uint16_t, kScanComp>(g, b, w, n_trials, num_sms, s, ev0, ev1, launches,      \
                                                          max_slots);                                            \
        return c16 ? launch_sweep_t<H, uint16_t, kScanFull>(g, b, w, n_trials, num_sms, s, ev0, ev1, launches,    \
                                                            max_slots)                                           \
                   : launch_sweep_t<H, uint32_t, kScanFull>(g, b, w, n_trials, num_sms, s, ev0, ev1, launches,    \
                                                            max_slots);                                          \
    }
    GRC_DISPATCH(1)
    GRC_DISPATCH(2)
    GRC_DISPATCH(3)
    GRC_DISPATCH(4)
#undef GRC_DISPATCH
    return cudaErrorInvalidValue;
}

namespace {
template <int HPL, typename CodeT>
cudaError_t launch_refine_list_t(const Geo &g, const ScoreBufs &b, const Work &w, int num_sms, cudaStream_t s) {
    const size_t smem_r = refine_smem_bytes(g.nrot, g.nhkl);
    int grid_r = 0;
    cudaError_t e = prep_launch(refine_list_kernel<HPL, CodeT>, smem_r, num_sms, (int64_t)num_sms * 4, &grid_r);
    if (e != cudaSuccess) return e;
    refine_list_kernel<HPL, CodeT><<<grid_r, kThreads, smem_r, s>>>(g, b, w);
    return cudaGetLastError();
}
}  // namespace

cudaError_t launch_refine_list(const Geo &g, const ScoreBufs &b, const Work &w, int num_sms, cudaStream_t s) {
    const int hpl = (g.nhkl + 31) / 32;
    const bool c16 = g.code_bits <= 16;
#define GRC_DISPATCH(H)                                                                                     \
    if (hpl == H)                                                                                           \
        return c16 ? launch_refine_list_t<H, uint16_t>(g, b, w, num_sms, s)                                 \
                   : launch_refine_list_t<H, uint32_t>(g, b, w, num_sms, s);
    GRC_DISPATCH(1)
    GRC_DISPATCH(2)
    GRC_DISPATCH(3)
    GRC_DISPATCH(4)
#undef GRC_DISPATCH
    return cudaErrorInvalidValue;
}

cudaError_t launch_pair(const Geo &g, const ScoreBufs &b, int64_t n, const SpotIndex &si, PairRec *out, int64_t cap,
                        unsigned long long *count, int num_sms, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    const size_t smem = pair_smem_bytes(g.nrot, g.nhkl);
    const void *fn = g.code_bits <= 16 ? (const void *)pair_kernel<uint16_t> : (const void *)pair_kernel<uint32_t>;
    cudaError_t e = allow_smem(fn, smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;  // CTAs of kPairThreads (occupancy_for counts kThreads-thread CTAs)
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kPairThreads, smem);
    if (e != cudaSuccess) return e;
    const int64_t resident = (int64_t)num_sms * (per_sm > 0 ? per_sm : 1);
    const int grid = (int)(n < resident ? n : resident);
    if (g.code_bits <= 16)
        pair_kernel<uint16_t><<<grid, kPairThreads, smem, s>>>(g, b, n, si, out, cap, count);
    else
        pair_kernel<uint32_t><<<grid, kPairThreads, smem, s>>>(g, b, n, si, out, cap, count);
    return cudaGetLastError();
}

}  // namespace grc
