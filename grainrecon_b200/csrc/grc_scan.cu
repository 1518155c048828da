// grc_scan.cu -- projection-window trial scan, one trial per warp at a time.
//
// The same work as the sweep of grc_score.cu (forward_comp.m:18-90 for every trial of a round,
// every CTA walking the projections window by window so the map pixels being read stay in L2),
// organised around the warp instead of the CTA:
//   * a warp takes one trial (slot) of the window at a time and first writes that trial's FP32
//     Gw table and window thresholds for all reflections into its own shared-memory table; the
//     prefilter keeps them in registers (lanes on reflections, as the sweep) and the per-item
//     landing reads them from the table instead of recomputing S*U*B*h and the window;
//   * the survivors of a trial go through a per-warp queue, 32 at a time, through the FP32 landing
//     chain with its FP64 band (landing_fp32 / landing_exact), and the queue is emptied at the end
//     of the trial, so every batch belongs to one trial: its pixels are counted in one register
//     of the warp (completeness-only mode: one bit of the packed hit mask per pixel) or in the
//     trial's 8-bit code histogram (full mode: Nr_simu, Nr_intersect and the exact median).
// Ambiguous items keep their trial in the FP64 queue, which is drained at the end of the window.
// Windows: up to 32 projections of 8-bit codes (full mode), up to 128 of the bit mask
// (completeness mode), each within the limits of shared memory and L2 (launch_scan_t).
// The decisions are those of the sweep and of the oracle: same prefilter margins, same FP32
// chain and band, same FP64 path.
#include <cuda_runtime.h>
#include <math_constants.h>
#include <stdint.h>

#include "grc_chain.cuh"
#include "grc_internal.h"

#ifndef GRC_SCAN_BLOCKS
#define GRC_SCAN_BLOCKS 3
#endif

namespace grc {
namespace {

constexpr int kScanSlots = 96;      // most trials a CTA holds in one round
constexpr int kScanSlotsBulk = 64;  // tile of multi-round work and of explicit voxel lists
constexpr int kScanWinMin = 8;
constexpr int kHistWords = 128;     // 256 u16 bins per slot, two per word
constexpr unsigned kAll = 0xffffffffu;

__device__ __forceinline__ int64_t scan_voxel_of(const Work &w, int64_t t) {
    if (w.trial_voxel) return (int64_t)w.trial_voxel[t];
    if (w.diag) return t;
    return t / w.n_or;
}

__device__ __forceinline__ int64_t scan_orient_of(const Work &w, int64_t t, int64_t v) {
    if (w.trial_orient) return (int64_t)w.trial_orient[t];
    return w.diag ? t : (t - v * w.n_or);
}

struct ScanSmem {
    RowF *rows;        // [rows_cap * nwin] omega rows of the window, vloc * nwin + wl
    float4 *hk;        // [nhkl] h as float
    uint32_t *hist;    // full mode: [slots * kHistWords]; completeness mode: [slots] packed counters
    float *subf;       // [slots * 12]
    double *subd;      // [slots * 9]
    int *vloc;         // [slots]
    int64_t *vglob;    // [slots]
    int64_t *vlist;    // [slots]
    float4 *wgw;       // [kWarps * nhkl] per-warp Gw table of the warp's trial: x, y, z, 1/|G|
    float4 *wwin;      // [kWarps * nhkl] its window thresholds (window_f)
    uint32_t *queue;   // [kWarps * kQueueCap]
    uint32_t *fqueue;  // [kWarps * kFallbackCap]
};

constexpr int kScanParts = 11;
__host__ __device__ inline size_t scan_smem_layout(int mode, int nhkl, int rows_cap, int slots, int nwin,
                                                   size_t *offs) {
    size_t o = 0, i = 0;
    auto put = [&](size_t bytes) {
        o = (o + 15) & ~size_t(15);
        offs[i++] = o;
        o += bytes;
    };
    put(sizeof(RowF) * rows_cap * nwin);
    put(sizeof(float4) * nhkl);
    put(sizeof(uint32_t) * slots * (mode == kScanFull ? kHistWords : 1));
    put(sizeof(float) * slots * 12);
    put(sizeof(double) * slots * 9);
    put(sizeof(int) * slots);
    put(sizeof(int64_t) * slots);
    put(sizeof(int64_t) * slots);
    put(sizeof(float4) * kWarps * nhkl);
    put(sizeof(float4) * kWarps * nhkl);
    put(sizeof(uint32_t) * kWarps * kQueueCap);
    o = (o + 15) & ~size_t(15);
    offs[i] = o;  // fqueue
    o += sizeof(uint32_t) * kWarps * kFallbackCap;
    return (o + 15) & ~size_t(15);
}

__device__ __forceinline__ ScanSmem scan_carve(unsigned char *base, int mode, int nhkl, int rows_cap, int slots,
                                               int nwin) {
    size_t offs[kScanParts + 1];
    scan_smem_layout(mode, nhkl, rows_cap, slots, nwin, offs);
    ScanSmem m;
    m.rows = (RowF *)(base + offs[0]);
    m.hk = (float4 *)(base + offs[1]);
    m.hist = (uint32_t *)(base + offs[2]);
    m.subf = (float *)(base + offs[3]);
    m.subd = (double *)(base + offs[4]);
    m.vloc = (int *)(base + offs[5]);
    m.vglob = (int64_t *)(base + offs[6]);
    m.vlist = (int64_t *)(base + offs[7]);
    m.wgw = (float4 *)(base + offs[8]);
    m.wwin = (float4 *)(base + offs[9]);
    m.queue = (uint32_t *)(base + offs[10]);
    m.fqueue = (uint32_t *)(base + offs[11]);
    return m;
}

template <int MODE, int HPL, int WIN>
__global__ void __launch_bounds__(kThreads, GRC_SCAN_BLOCKS)
    scan_kernel(Geo g, ScoreBufs b, Work w, int64_t round_base, int64_t n_trials, int rows_cap, int slots) {
    const int64_t cta_base = round_base + (int64_t)blockIdx.x * slots;
    if (cta_base >= n_trials) return;
    const int nslot = (int)min((int64_t)slots, n_trials - cta_base);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const ScanSmem sm = scan_carve(smem_raw, MODE, g.nhkl, rows_cap, slots, WIN);
    __shared__ int s_nv, s_next;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const unsigned lt = (1u << lane) - 1u;
    uint32_t *wq = sm.queue + warp * kQueueCap;
    uint32_t *fq = sm.fqueue + warp * kFallbackCap;
    float4 *gwt = sm.wgw + warp * g.nhkl;
    float4 *wnt = sm.wwin + warp * g.nhkl;

    // ---- set-up: per-slot S*U*B, voxels, zeroed counters
    if (tid < nslot) {
        const int64_t t = cta_base + tid;
        const int64_t v = scan_voxel_of(w, t);
        const int64_t o = scan_orient_of(w, t, v);
        double SUB[9];
        sub_matrix(g, b.U + 9 * o, SUB);
#pragma unroll
        for (int i = 0; i < 9; ++i) {
            sm.subd[9 * tid + i] = SUB[i];
            sm.subf[12 * tid + i] = (float)SUB[i];
        }
        sm.vglob[tid] = v;
    }
    for (int i = tid; i < slots * (MODE == kScanFull ? kHistWords : 1); i += kThreads) sm.hist[i] = 0;
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
    const uint32_t pw32 = (uint32_t)pw;

    for (int w0 = 0; w0 < g.nrot; w0 += WIN) {
        const int nw = min(WIN, g.nrot - w0);
        // ---- omega rows of this window for every voxel of the round
        for (int i = tid; i < nv * nw; i += kThreads) {
            const int vl = i / nw, wl = i - vl * nw;
            sm.rows[vl * WIN + wl] = row_f32(g, omega_row(g, b.rot_cs[w0 + wl], b.vpos + 3 * sm.vlist[vl]));
        }
        if (tid == 0) s_next = 0;
        __syncthreads();

        const uint8_t *wcodes = MODE == kScanFull ? b.codes8 + (int64_t)w0 * g.plane : nullptr;
        const uint32_t *wbits = MODE == kScanComp ? b.bits + (int64_t)w0 * pw : nullptr;
        int fn = 0;  // ambiguous items of this warp (any of its trials), drained at the window end

        // FP64 path of one ambiguous item: counted at once (shared atomics; these items are rare)
        auto exact = [&](uint32_t item, bool valid) {
            const int s2 = (int)(item >> 16), wl = (int)((item >> 8) & 255u), ih = (int)(item & 255u);
            if (!valid) return;
            const int64_t r64 =
                landing_exact(b.geo, b.rot_cs, b.vpos + 3 * sm.vglob[s2], b.hkl, sm.subd + 9 * s2, w0 + wl, ih);
            if (r64 < 0) return;
            if (MODE == kScanComp) {
                const int64_t iw = w0 + wl, ip = r64 - iw * g.plane;
                const uint32_t word = __ldg(b.bits + iw * pw + (ip >> 5));
                atomicAdd(&sm.hist[s2], 1u + (((word >> (ip & 31)) & 1u) << 16));
            } else {
                const uint32_t code = __ldg(b.codes8 + r64);
                atomicAdd(&sm.hist[s2 * kHistWords + (code >> 1)], 1u << ((code & 1u) * 16));
            }
        };
        auto drain_exact = [&](bool all) {
            while (fn >= 32 || (all && fn > 0)) {
                const int take = fn >= 32 ? 32 : fn;
                fn -= take;
                const bool v2 = lane < take;
                const uint32_t it2 = v2 ? fq[fn + lane] : 0u;
                __syncwarp();
                exact(it2, v2);
                __syncwarp();
            }
        };

        // slots are handed out one at a time, so the warps of a CTA reach the end-of-window
        // barrier together however unevenly the selected reflections fall on the slots
        for (;;) {
            int s = 0;
            if (lane == 0) s = atomicAdd(&s_next, 1);
            s = __shfl_sync(kAll, s, 0);
            if (s >= nslot) break;
            const float *sf = sm.subf + 12 * s;
            // ---- the trial's Gw table (shared, for the landings) and prefilter (registers)
            float gx[HPL], gy[HPL], gz[HPL], lo[HPL], hi[HPL];
#pragma unroll
            for (int j = 0; j < HPL; ++j) {
                const int ih = lane + 32 * j;
                gx[j] = gy[j] = gz[j] = 0.f;
                lo[j] = CUDART_INF_F;
                hi[j] = -CUDART_INF_F;
                if (ih < g.nhkl) {
                    const float4 gv = gw_of(sf, sm.hk[ih]);
                    const float4 wv = window_f(g, gv);
                    gwt[ih] = gv;
                    wnt[ih] = wv;
                    gx[j] = gv.x;
                    gy[j] = gv.y;
                    gz[j] = gv.z;
                    lo[j] = wv.x;
                    hi[j] = wv.y;
                }
            }
            __syncwarp();
            const RowF *vr = sm.rows + sm.vloc[s] * WIN;
            // completeness mode: the lane's share of this trial's counts in this window, packed as
            // the shared counter (Nr_simu low, Nr_intersect high 16 bits) and summed over the warp
            // once per trial and window
            uint32_t cnt = 0;
            // a selected pixel is read when its batch is evaluated and counted after the next batch
            // has been computed, so the gather's latency overlaps the landing arithmetic; pend_bit
            // is the pixel's bit (completeness) or 0 (full), -1 when the lane has none
            int pend_bit = -1;
            uint32_t pend_val = 0;
            auto apply_pending = [&]() {
                if (MODE == kScanComp) {
                    const bool sel = pend_bit >= 0;
                    const bool hit = sel && ((pend_val >> pend_bit) & 1u);
                    cnt += (uint32_t)sel + ((uint32_t)hit << 16);
                } else if (pend_bit >= 0) {
                    atomicAdd(&sm.hist[s * kHistWords + (pend_val >> 1)], 1u << ((pend_val & 1u) * 16));
                }
                pend_bit = -1;
            };
            auto fast = [&](uint32_t item, bool valid) {
                const int wl = (int)(item >> 8), ih = (int)(item & 255u);
                int ip = -1;
                if (valid) {
                    const float4 gv = gwt[ih];
                    const float4 wv = wnt[ih];
                    ip = landing_fp32(g, vr[wl], gv, wv.z, wv.w);
                }
                const unsigned m = __ballot_sync(kAll, ip == -2);
                if (m) {  // ambiguous items (rare) join the FP64 queue
                    if (ip == -2) fq[fn + __popc(m & lt)] = ((uint32_t)s << 16) | item;
                    fn += __popc(m);
                }
                uint32_t val = 0;
                if (ip >= 0) {
                    // offsets within the window fit 32 bits: WIN * plane < 2^31 for the codes
                    // (launch_scan_t) and 8 * plane < 2^31 for the words (scan_round_trials)
                    if (MODE == kScanComp)
                        val = __ldg(wbits + ((uint32_t)wl * pw32 + ((uint32_t)ip >> 5)));
                    else
                        val = __ldg(wcodes + ((uint32_t)wl * (uint32_t)g.plane + (uint32_t)ip));
                }
                apply_pending();
                pend_bit = ip >= 0 ? (MODE == kScanComp ? (ip & 31) : 0) : -1;
                pend_val = val;
            };
            int qn = 0;
            for (int wl = 0; wl < nw; ++wl) {
                const float4 kwv = reinterpret_cast<const float4 *>(vr + wl)[3];
#pragma unroll
                for (int j = 0; j < HPL; ++j) {
                    const float t = -fmaf(kwv.x, gx[j], fmaf(kwv.y, gy[j], kwv.z * gz[j]));
                    const bool pass = (t > lo[j]) && (t < hi[j]);
                    const unsigned bm = __ballot_sync(kAll, pass);
                    if (pass) wq[qn + __popc(bm & lt)] = ((uint32_t)wl << 8) | (uint32_t)(lane + 32 * j);
                    qn += __popc(bm);
                }
                __syncwarp();
                while (qn >= 32) {
                    qn -= 32;
                    const uint32_t item = wq[qn + lane];
                    __syncwarp();
                    fast(item, true);
                    __syncwarp();
                    drain_exact(false);
                }
            }
            if (qn > 0) {  // the trial's last, partial batch: every batch holds one trial
                const bool valid = lane < qn;
                const uint32_t item = valid ? wq[lane] : 0u;
                __syncwarp();
                fast(item, valid);
                __syncwarp();
                drain_exact(false);
            }
            apply_pending();
            if (MODE == kScanComp) {
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(kAll, cnt, o);
                if (lane == 0) atomicAdd(&sm.hist[s], cnt);
            }
        }
        drain_exact(true);
        __syncthreads();  // rows are rebuilt for the next window
    }

    // ---- finalize
    if constexpr (MODE == kScanFull) {
        for (int s = warp; s < nslot; s += kWarps) hist8_finish(g, b, sm.hist + s * kHistWords, cta_base + s);
    } else {
        for (int base = warp * 32; base < nslot; base += kWarps * 32) {
            const int s = base + lane;
            const bool in = s < nslot;
            const int64_t t = cta_base + s;
            int simu = 0, inter = 0;
            if (in) {
                const uint32_t c = sm.hist[s];
                simu = (int)(c & 0xffffu);
                inter = (int)(c >> 16);
                TrialRes r;
                r.simu = simu;
                r.inter = inter;
                r.median = CUDART_NAN;  // not computed in this mode
                b.res[t] = r;
            }
            if (b.group_key) fold_group_key(b, in, t, simu, inter);
        }
    }
}

template <int MODE, int HPL>
cudaError_t launch_scan_t(const Geo &g, const ScoreBufs &b, const Work &w, int64_t n_trials, int num_sms,
                          cudaStream_t s, cudaEvent_t ev0, cudaEvent_t ev1, int *launches, int max_slots) {
    // Tiles as the sweep: kScanSlotsBulk trials per CTA; an implicit seeding list may take up to
    // kScanSlots when that fits the call into one round; explicit lists keep one row set per
    // voxel-run start of their aligned 32-trial blocks.
    const bool explicit_voxels = w.trial_voxel || w.diag || w.n_or <= 0;
    const bool caller_tile = max_slots >= 1 && max_slots <= kScanSlots;
    if (!caller_tile) max_slots = kScanSlotsBulk;
    auto rows_for = [&](int sl) {
        int rc = (int)(w.n_or >= sl ? 2 : (w.n_or > 0 ? sl / w.n_or + 2 : sl));
        if (explicit_voxels) rc = w.starts_per_32 > 0 ? 1 + ((sl + 31) / 32 + 1) * w.starts_per_32 : sl;
        return rc > sl ? sl : rc;
    };
    size_t offs[kScanParts + 1];
    using ScanFn = void (*)(Geo, ScoreBufs, Work, int64_t, int64_t, int, int);
    const ScanFn k8 = scan_kernel<MODE, HPL, kScanWinMin>;
    const size_t smem_max = scan_smem_layout(MODE, g.nhkl, rows_for(max_slots), max_slots, kScanWinMin, offs);
    int per_sm = 0;
    cudaError_t e = occupancy_for((const void *)k8, smem_max, &per_sm);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    const int64_t grid = (int64_t)per_sm * num_sms;
    if (!caller_tile && !explicit_voxels && n_trials > grid * max_slots && n_trials <= grid * kScanSlots) {
        int per_sm1 = 0;
        const size_t smem1 = scan_smem_layout(MODE, g.nhkl, rows_for(kScanSlots), kScanSlots, kScanWinMin, offs);
        if (occupancy_for((const void *)k8, smem1, &per_sm1) == cudaSuccess && per_sm1 == per_sm)
            max_slots = kScanSlots;
    }
    const int64_t rounds = (n_trials + grid * max_slots - 1) / (grid * max_slots);
    int slots = (int)((n_trials + rounds * grid - 1) / (rounds * grid));
    if (slots < 1) slots = 1;
    const int rows_cap = rows_for(slots);
    // the widest projection window whose rows keep the grid's CTAs per SM: up to 128 projections
    // for the bit mask of a seeding scan (one-seed Al rounds 1.641 / 1.567 / 1.573 ms at 32 / 64 /
    // 128, 64-seed calls 103.9 / 98.7 / 97.1 ms), 32 or 16 for the 8-bit codes (32 projections of
    // 2048^2 codes are already about the size of L2; 16 ran 6-8 % slower), else 8
    ScanFn kern = k8;
    size_t smem = scan_smem_layout(MODE, g.nhkl, rows_cap, slots, kScanWinMin, offs);
    bool refused = false;
    auto window_kernel = [](int cand) -> ScanFn {
        if constexpr (MODE == kScanComp) {
            if (cand == 128) return scan_kernel<MODE, HPL, 128>;
            if (cand == 64) return scan_kernel<MODE, HPL, 64>;
        }
        return cand == 32 ? (ScanFn)scan_kernel<MODE, HPL, 32> : (ScanFn)scan_kernel<MODE, HPL, 16>;
    };
    // Explicit trial lists in completeness mode (the seeding refine's grids) take at most 64: the
    // refine of 16 Al seeds took 0.223 s with 64-projection windows, 0.234 s with 32 and
    // 0.246-0.255 s with 128.
    const bool wide = MODE == kScanComp;
    const int kCands = wide ? 4 : 2;
    const int cands_wide[4] = {explicit_voxels ? 64 : 128, 64, 32, 16}, cands_narrow[2] = {32, 16};
    const int *cands = wide ? cands_wide : cands_narrow;
    // the bit-mask window stays within 3/4 of L2 (Al 2048^2 on 126 MB: 128 projections = 67 MB,
    // fastest; 256 = 134 MB ran 30% slower)
    int64_t l2_budget = 0;
    if (MODE == kScanComp) {
        int dev = 0, l2 = 0;
        if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, dev) == cudaSuccess)
            l2_budget = (int64_t)l2 * 3 / 4;
        else
            cudaGetLastError();  // no L2 size: windows of at most 32 projections
    }
    for (int ci = 0; ci < kCands; ++ci) {
        const int cand = cands[ci];
        if (MODE == kScanComp && cand > 32 && (int64_t)cand * b.plane_words * 4 > l2_budget) continue;
        if (MODE == kScanFull && (int64_t)cand * g.plane > 2147483647LL) continue;
        const ScanFn kc = window_kernel(cand);
        const size_t smem_c = scan_smem_layout(MODE, g.nhkl, rows_cap, slots, cand, offs);
        int per_c = 0;
        if (occupancy_for((const void *)kc, smem_c, &per_c) != cudaSuccess) {
            refused = true;
            continue;
        }
        if (per_c >= per_sm) {
            kern = kc;
            smem = smem_c;
            break;
        }
    }
    if (refused) cudaGetLastError();  // a refused window query is not an error of this launch
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
    if (MODE == kScanFull) {
        e = launch_refine_list(g, b, w, num_sms, s);
        if (e != cudaSuccess) return e;
        ++*launches;
    }
    return cudaGetLastError();
}

template <typename CodeT>
__global__ void pack_bits_k(const CodeT *codes, int64_t plane, int64_t nrot, uint32_t n_hit, int64_t pw,
                            uint32_t *bits) {
    // one thread per bit of the padded layout; a warp covers one 32-bit word
    const int64_t per_plane = pw * 32, total = nrot * per_plane;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;  // a multiple of 32
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
        const int64_t iw = i / per_plane, p = i - iw * per_plane;
        const bool hit = p < plane && (uint32_t)codes[iw * plane + p] < n_hit;
        const unsigned m = __ballot_sync(kAll, hit);
        if ((threadIdx.x & 31) == 0) bits[i >> 5] = m;
    }
}

// One warp per group: the first maximum of completeness over the group's trials.
__global__ void group_argmax_k(const TrialRes *res, int64_t n_trials, int64_t gsize, unsigned long long *keys) {
    const int lane = threadIdx.x & 31;
    const int64_t n_groups = (n_trials + gsize - 1) / gsize;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t grp = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); grp < n_groups; grp += warps) {
        const int64_t t0 = grp * gsize, n = min(gsize, n_trials - t0);
        unsigned long long key = 0ull;
        for (int64_t i = lane; i < n; i += 32) {
            const TrialRes r = res[t0 + i];
            const unsigned long long k = group_key_of(r.simu, r.inter, i);
            key = k > key ? k : key;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long y = shfl_xor_u64(key, o);
            key = y > key ? y : key;
        }
        if (lane == 0) atomicMax(keys + grp, key);
    }
}

__global__ void group_decode_k(const unsigned long long *keys, int64_t n_groups, int32_t *best, float *best_c) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_groups; i += (int64_t)gridDim.x * blockDim.x) {
        const unsigned long long k = keys[i];
        const uint32_t hi = (uint32_t)(k >> 32), lo = (uint32_t)k;
        if (best) best[i] = (int32_t)(0xffffffffu - lo);
        if (best_c) best_c[i] = hi == 0u ? CUDART_NAN_F : __uint_as_float(hi - 1u);
    }
}

// Spot pixels of a packed mask back to bytes: mask[iw*plane + p] = bit p of projection iw.
__global__ void unpack_bits_k(const uint32_t *bits, int64_t plane, int64_t nrot, int64_t pw, uint8_t *mask) {
    const int64_t n = nrot * plane;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t iw = i / plane, p = i - iw * plane;
        mask[i] = (uint8_t)((bits[iw * pw + (p >> 5)] >> (p & 31)) & 1u);
    }
}

}  // namespace

cudaError_t launch_unpack_bits(const uint32_t *bits, int64_t plane, int64_t nrot, int64_t plane_words, uint8_t *mask,
                               cudaStream_t s) {
    const int64_t n = nrot * plane;
    if (n <= 0) return cudaSuccess;
    const int64_t want = (n + 255) / 256;
    unpack_bits_k<<<(int)(want < 65535 * 8 ? want : 65535 * 8), 256, 0, s>>>(bits, plane, nrot, plane_words, mask);
    return cudaGetLastError();
}

cudaError_t launch_group_argmax(const TrialRes *res, int64_t n_trials, int64_t gsize, unsigned long long *keys,
                                cudaStream_t s) {
    if (n_trials <= 0 || gsize <= 0) return cudaSuccess;
    const int64_t n_groups = (n_trials + gsize - 1) / gsize;
    const int64_t want = (n_groups + 7) / 8;
    const int blocks = (int)(want < 65535 * 4 ? want : 65535 * 4);
    group_argmax_k<<<blocks, 256, 0, s>>>(res, n_trials, gsize, keys);
    return cudaGetLastError();
}

cudaError_t launch_group_decode(const unsigned long long *keys, int64_t n_groups, int32_t *best, float *best_c,
                                cudaStream_t s) {
    if (n_groups <= 0) return cudaSuccess;
    const int64_t want = (n_groups + 255) / 256;
    const int blocks = (int)(want < 65535 ? want : 65535);
    group_decode_k<<<blocks, 256, 0, s>>>(keys, n_groups, best, best_c);
    return cudaGetLastError();
}

int64_t scan_round_trials(const Geo &g, int num_sms) {
    // 16-bit histogram bins (full mode) and 13-bit items; hit codes below the saturation code
    if (g.n_hit >= 255u || g.nhkl > 128 || (int64_t)g.nrot * g.nhkl > 65535 ||
        (int64_t)kScanWinMin * g.plane > 2147483647LL)
        return 0;
    return (int64_t)num_sms * GRC_SCAN_BLOCKS * kScanSlotsBulk;
}

cudaError_t launch_scan(const Geo &g, const ScoreBufs &b, const Work &w, int64_t n_trials, int num_sms, int mode,
                        cudaStream_t s, cudaEvent_t ev0, cudaEvent_t ev1, int *launches, int max_slots) {
    const int hpl = (g.nhkl + 31) / 32;
    if (mode == kScanComp && !b.bits) return cudaErrorInvalidValue;
#define GRC_DISPATCH(H)                                                                                    \
    if (hpl == H)                                                                                          \
        return mode == kScanComp                                                                           \
                   ? launch_scan_t<kScanComp, H>(g, b, w, n_trials, num_sms, s, ev0, ev1, launches, max_slots) \
                   : launch_scan_t<kScanFull, H>(g, b, w, n_trials, num_sms, s, ev0, ev1, launches, max_slots);
    GRC_DISPATCH(1)
    GRC_DISPATCH(2)
    GRC_DISPATCH(3)
    GRC_DISPATCH(4)
#undef GRC_DISPATCH
    return cudaErrorInvalidValue;
}

cudaError_t launch_pack_bits(const void *codes, int code_bytes, int64_t plane, int64_t nrot, uint32_t n_hit,
                             int64_t plane_words, uint32_t *bits, cudaStream_t s) {
    const int64_t total = nrot * plane_words * 32;
    const int threads = 256;
    const int64_t want = (total + threads - 1) / threads;
    const int blocks = (int)(want < 65535 * 8 ? want : 65535 * 8);
    if (code_bytes == 1)
        pack_bits_k<uint8_t><<<blocks, threads, 0, s>>>((const uint8_t *)codes, plane, nrot, n_hit, plane_words, bits);
    else if (code_bytes == 2)
        pack_bits_k<uint16_t><<<blocks, threads, 0, s>>>((const uint16_t *)codes, plane, nrot, n_hit, plane_words,
                                                          bits);
    else
        pack_bits_k<uint32_t><<<blocks, threads, 0, s>>>((const uint32_t *)codes, plane, nrot, n_hit, plane_words,
                                                          bits);
    return cudaGetLastError();
}

}  // namespace grc
