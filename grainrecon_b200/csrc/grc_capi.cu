// grc_capi.cu -- the C ABI (include/grainrecon_b200.h): context, resident distance
// map, geometry cache and the drop-in entries replacing GrainRecon's CUDA MEX calls.
#include <cub/cub.cuh>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <new>
#include <vector>

#include "grainrecon_b200.h"
#include "grc_fit.h"
#include "grc_internal.h"

namespace {

struct DevBuf {
    void *p = nullptr;
    size_t cap = 0;
};

// Trials per work item of a seeding scan: one omega table serves this many orientations.
constexpr int kSeedChunk = 16;

}  // namespace

struct grc_ctx {
    int device = 0;
    int num_sms = 0;
    cudaStream_t stream = nullptr;
    std::mutex mu;
    std::string err;
    double opt_dety0 = NAN, opt_detz0 = NAN, opt_thr = 0.5;
    bool has_geo = false;
    std::vector<float> geo_key;
    grc::Geo geo{};
    bool has_masks = false;
    grc::MapCodes mc{};
    int64_t mz = 0, my = 0, mrot = 0;
    std::vector<float> h_vals;
    DevBuf fgeo, fne, ftrial, fcost0, fcost1, fimp, fhw, geo_dev, rot_cs, hkl, pos, U, res, tvoxel, rlist, in1, in2, in3, out, items, torient, counts, offsets, tmp, counter, p1, bad, nm, sp_keys, sp_ids, sp_keys2, sp_ids2, cell_cnt, cell_off, pr_raw, pr_keys, pr_keys2, pr_ids, pr_ids2, pcount, nmloop;
    grc::Geo *geo_pinned = nullptr;  // staging of the per-launch geometry copy
    grc::Geo geo_up{};               // the geometry geo_dev holds (valid when geo_up_ok)
    bool geo_up_ok = false;
    int *nm_active = nullptr;        // pinned: seeds still running in the orientation fit
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    bool timing = false;
    bool timed_last = false;
    int force_path = 0;  // 0 = by size, 1 = per-trial kernel, 2 = CTA sweep, 3 = warp scan
    bool median = true;  // seeding-scan entries: false = completeness only (bit-packed mask)
    DevBuf bits, gkey;   // bit-packed hit mask of the resident map; per-group argmax keys
    DevBuf sgrid, sgrid32, stv, sto, sbest;  // seeding-stage grids, trial lists, grid maxima
    bool bits_ok = false;
    uint32_t bits_hit = 0;
    uint64_t map_key = 0;  // content key of the resident map (grc_upload_masks_if_changed), 0 = none
    int64_t plane_words = 0;
    grc_stats stats{};
};

namespace {

int fail(grc_ctx *c, int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (c) c->err = buf;
    return code;
}

#define CU(x)                                                                                      \
    do {                                                                                           \
        cudaError_t e_ = (x);                                                                      \
        if (e_ != cudaSuccess) return fail(ctx, GRC_ECUDA, "%s: %s", #x, cudaGetErrorString(e_)); \
    } while (0)

#define TRY(x)                 \
    do {                       \
        int r_ = (x);          \
        if (r_ != GRC_OK) return r_; \
    } while (0)

int ensure(grc_ctx *ctx, DevBuf &b, size_t bytes) {
    if (bytes == 0) bytes = 16;
    if (b.cap >= bytes) return GRC_OK;
    const size_t want = std::max(bytes, b.cap + b.cap / 2);
    CU(cudaStreamSynchronize(ctx->stream));
    if (b.p) CU(cudaFree(b.p));
    b.p = nullptr;
    b.cap = 0;
    cudaError_t e = cudaMalloc(&b.p, want);
    if (e != cudaSuccess) return fail(ctx, GRC_ECUDA, "cudaMalloc(%zu bytes): %s", want, cudaGetErrorString(e));
    b.cap = want;
    return GRC_OK;
}

bool is_device_ptr(const void *p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

bool is_int(float v) { return std::isfinite(v) && std::floor(v) == v; }

// A *_device entry hands its buffers straight to kernels: a host pointer there would fault on
// the GPU, so it is refused here.  NULL passes (the callers check NULL with their own message).
int need_device(grc_ctx *ctx, const void *p, const char *what) {
    if (p && !is_device_ptr(p)) return fail(ctx, GRC_EINVAL, "%s is not device memory", what);
    return GRC_OK;
}

void refresh_hit(grc_ctx *ctx) {
    if (!ctx->has_masks) return;
    const double thr = ctx->opt_thr;
    size_t n = 0;
    while (n < ctx->h_vals.size() && (double)ctx->h_vals[n] <= thr) ++n;
    ctx->geo.n_hit = (uint32_t)n;
    if (ctx->bits_hit != ctx->geo.n_hit) ctx->bits_ok = false;  // the packed mask follows the threshold
    ctx->geo.n_vals = (uint32_t)std::max<int64_t>(1, ctx->mc.n_distinct);
    int bits = 0;
    while (bits < 32 && (int64_t(1) << bits) < ctx->mc.n_distinct) ++bits;
    ctx->geo.code_bits = bits;
}

void apply_options(grc_ctx *ctx) {
    grc::Geo &g = ctx->geo;
    g.dety0 = std::isnan(ctx->opt_dety0) ? g.detysize / 2.0 + 0.5 : ctx->opt_dety0;
    g.detz0 = std::isnan(ctx->opt_detz0) ? g.detzsize / 2.0 + 0.5 : ctx->opt_detz0;
    for (int i = 0; i < 9; ++i) g.Rf[i] = (float)g.R[i];
    g.Ruf[0] = (float)(g.R[4] / g.pxy);
    g.Ruf[1] = (float)(g.R[7] / g.pxy);
    g.Rvf[0] = (float)(g.R[5] / g.pxz);
    g.Rvf[1] = (float)(g.R[8] / g.pxz);
    g.dety0f = (float)g.dety0;
    g.detz0f = (float)g.detz0;
    g.rpxyf = (float)(1.0 / g.pxy);
    g.rpxzf = (float)(1.0 / g.pxz);
    g.bsy0f = (float)g.bsy0;
    g.bsy1f = (float)g.bsy1;
    g.bsz0f = (float)g.bsz0;
    g.bsz1f = (float)g.bsz1;
    g.lo4pif = (float)(g.lmin * 0.25 / 3.14159265358979323846);
    g.hi4pif = (float)(g.lmax * 0.25 / 3.14159265358979323846);
    g.cbmaxf = (float)g.cbmax;
    refresh_hit(ctx);
}

int set_geometry(grc_ctx *ctx, const float *S, const float *B, const float *hkl, const float *rot,
                 const float *R, const float *param) {
    if (!S || !B || !hkl || !rot || !R || !param) return fail(ctx, GRC_EINVAL, "geometry: NULL argument");
    for (int i = 0; i < 20; ++i)
        if (!std::isfinite(param[i])) return fail(ctx, GRC_EINVAL, "param(%d) is not finite", i + 1);
    if (!is_int(param[0]) || param[0] < 1) return fail(ctx, GRC_EINVAL, "param(1)=nr_hkl must be a positive integer");
    if (!is_int(param[1]) || param[1] < 1) return fail(ctx, GRC_EINVAL, "param(2)=nr_rot must be a positive integer");
    if (param[0] > GRC_MAX_NHKL)
        return fail(ctx, GRC_ECAPACITY, "nr_hkl=%g exceeds GRC_MAX_NHKL=%d", param[0], GRC_MAX_NHKL);
    if (param[1] > GRC_MAX_NROT)
        return fail(ctx, GRC_ECAPACITY, "nr_rot=%g exceeds GRC_MAX_NROT=%d", param[1], GRC_MAX_NROT);
    if (!is_int(param[10]) || !is_int(param[11]) || param[10] < 1 || param[11] < 1)
        return fail(ctx, GRC_EINVAL, "detysize/detzsize must be positive integers");
    if (param[10] > 1e6f || param[11] > 1e6f || (double)param[10] * (double)param[11] > 2147483647.0)
        return fail(ctx, GRC_ECAPACITY, "detector %gx%g: at most 10^6 pixels per side and 2^31-1 in all",
                    param[10], param[11]);
    if (!(param[8] > 0) || !(param[9] > 0)) return fail(ctx, GRC_EINVAL, "pixel sizes must be positive");
    const int nhkl = (int)param[0], nrot = (int)param[1];
    std::vector<float> key;
    key.reserve(47 + 3 * nhkl + nrot);
    key.insert(key.end(), S, S + 9);
    key.insert(key.end(), B, B + 9);
    key.insert(key.end(), R, R + 9);
    key.insert(key.end(), param, param + 20);
    key.insert(key.end(), hkl, hkl + 3 * nhkl);
    key.insert(key.end(), rot, rot + nrot);
    for (float v : key)
        if (!std::isfinite(v)) return fail(ctx, GRC_EINVAL, "geometry array holds a non-finite value");
    if (ctx->has_geo && key.size() == ctx->geo_key.size() &&
        std::memcmp(key.data(), ctx->geo_key.data(), key.size() * sizeof(float)) == 0) {
        apply_options(ctx);
        return GRC_OK;
    }
    grc::Geo g{};
    g.nhkl = nhkl;
    g.nrot = nrot;
    g.lss = param[2]; g.lsd = param[3]; g.p0y = param[4]; g.p0z = param[5];
    g.dety00 = param[6]; g.detz00 = param[7]; g.pxy = param[8]; g.pxz = param[9];
    g.detysize = (int)param[10]; g.detzsize = (int)param[11];
    g.bsy0 = param[12]; g.bsy1 = param[13]; g.bsz0 = param[14]; g.bsz1 = param[15];
    g.lmin = param[17]; g.lmax = param[18]; g.rao = param[19];
    const double pi = 3.14159265358979323846;
    const double bmax = (90.0 + (double)param[16] * 4.0) / 180.0 * pi;  // forward_comp.m:61
    g.cbmax = bmax <= pi ? std::cos(bmax) : -2.0;
    for (int i = 0; i < 9; ++i) {
        g.S[i] = S[i];
        g.B[i] = B[i];
        g.R[i] = R[i];
    }
    g.plane = (int64_t)g.detysize * g.detzsize;
    std::vector<double2> cs(nrot);
    for (int i = 0; i < nrot; ++i) {
        const double w = (double)rot[i] * pi / 180.0;  // forward_comp.m:19
        cs[i] = make_double2(std::cos(w), std::sin(w));
    }
    std::vector<double> h(3 * nhkl);
    for (int i = 0; i < 3 * nhkl; ++i) h[i] = hkl[i];
    TRY(ensure(ctx, ctx->rot_cs, sizeof(double2) * nrot));
    TRY(ensure(ctx, ctx->hkl, sizeof(double) * 3 * nhkl));
    CU(cudaMemcpyAsync(ctx->rot_cs.p, cs.data(), sizeof(double2) * nrot, cudaMemcpyHostToDevice, ctx->stream));
    CU(cudaMemcpyAsync(ctx->hkl.p, h.data(), sizeof(double) * 3 * nhkl, cudaMemcpyHostToDevice, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    ctx->geo = g;
    ctx->geo_key.swap(key);
    ctx->has_geo = true;
    apply_options(ctx);
    return GRC_OK;
}

int upload_device_map(grc_ctx *ctx, const float *d_map, int64_t dz, int64_t dy, int64_t nrot) {
    const int64_t n = dz * dy * nrot;
    grc::MapCodes mc{};
    int bad = 0;
    cudaError_t e = grc::encode_map(d_map, n, ctx->stream, &mc, &bad);
    if (e != cudaSuccess) return fail(ctx, GRC_ECUDA, "distance-map coding: %s", cudaGetErrorString(e));
    if (bad) return fail(ctx, GRC_EINVAL, "distance map holds NaN values");
    std::vector<float> hv((size_t)mc.n_distinct);
    if (mc.n_distinct > 0) {
        e = cudaMemcpy(hv.data(), mc.vals, sizeof(float) * mc.n_distinct, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) {
            cudaFree(mc.codes);
            cudaFree(mc.codes8);
            cudaFree(mc.vals);
            return fail(ctx, GRC_ECUDA, "value table copy: %s", cudaGetErrorString(e));
        }
    }
    if (ctx->has_masks) {
        cudaFree(ctx->mc.codes);
        cudaFree(ctx->mc.codes8);
        cudaFree(ctx->mc.vals);
    }
    ctx->mc = mc;
    ctx->bits_ok = false;  // packed again from the new codes when first needed
    ctx->map_key = 0;      // an upload that came without a key
    ctx->h_vals.swap(hv);
    ctx->mz = dz;
    ctx->my = dy;
    ctx->mrot = nrot;
    ctx->has_masks = true;
    refresh_hit(ctx);
    return GRC_OK;
}

int upload_host_map(grc_ctx *ctx, const float *map, int64_t dz, int64_t dy, int64_t nrot) {
    if (!map) return fail(ctx, GRC_EINVAL, "proj_bin_bw is NULL");
    if (dz < 1 || dy < 1 || nrot < 1) return fail(ctx, GRC_EINVAL, "distance-map dimensions must be positive");
    const int64_t n = dz * dy * nrot;
    float *d_map = nullptr;
    cudaError_t e = cudaMalloc(&d_map, sizeof(float) * n);
    if (e != cudaSuccess) return fail(ctx, GRC_ECUDA, "cudaMalloc(map): %s", cudaGetErrorString(e));
    // chunked copy keeps the pageable staging small
    const int64_t chunk = int64_t(1) << 26;
    for (int64_t s = 0; s < n && e == cudaSuccess; s += chunk) {
        const int64_t c = std::min(chunk, n - s);
        e = cudaMemcpyAsync(d_map + s, map + s, sizeof(float) * c, cudaMemcpyHostToDevice, ctx->stream);
    }
    if (e != cudaSuccess) {
        cudaFree(d_map);
        return fail(ctx, GRC_ECUDA, "map upload: %s", cudaGetErrorString(e));
    }
    int r = upload_device_map(ctx, d_map, dz, dy, nrot);
    cudaStreamSynchronize(ctx->stream);
    cudaFree(d_map);
    return r;
}

int check_ready(grc_ctx *ctx) {
    if (!ctx->has_geo) return fail(ctx, GRC_EINVAL, "no geometry set");
    if (!ctx->has_masks) return fail(ctx, GRC_ENOMASK, "no distance map resident and none passed");
    const grc::Geo &g = ctx->geo;
    if (ctx->mz != g.detzsize || ctx->my != g.detysize || ctx->mrot != g.nrot)
        return fail(ctx, GRC_EINVAL,
                    "distance map is %lld x %lld x %lld (detz x dety x nrot) but param says %d x %d x %d",
                    (long long)ctx->mz, (long long)ctx->my, (long long)ctx->mrot, g.detzsize, g.detysize, g.nrot);
    return GRC_OK;
}

// Bit-packed hit mask of the resident map (bit = code < n_hit), built on the device the first time a
// completeness-only scan needs it and again after a new map or threshold: 1 bit per pixel,
// plane_words 32-bit words per projection (a 16-byte multiple).
int ensure_bits(grc_ctx *ctx) {
    const grc::Geo &g = ctx->geo;
    if (ctx->bits_ok && ctx->bits_hit == g.n_hit) return GRC_OK;
    const int64_t pw = (g.plane + 127) / 128 * 4;
    TRY(ensure(ctx, ctx->bits, sizeof(uint32_t) * pw * g.nrot));
    if (g.n_hit < 255u)
        CU(grc::launch_pack_bits(ctx->mc.codes8, 1, g.plane, g.nrot, g.n_hit, pw, (uint32_t *)ctx->bits.p,
                                 ctx->stream));
    else
        CU(grc::launch_pack_bits(ctx->mc.codes, g.code_bits <= 16 ? 2 : 4, g.plane, g.nrot, g.n_hit, pw,
                                 (uint32_t *)ctx->bits.p, ctx->stream));
    ctx->plane_words = pw;
    ctx->bits_hit = g.n_hit;
    ctx->bits_ok = true;
    return GRC_OK;
}

grc::ScoreBufs bufs(grc_ctx *ctx) {
    grc::ScoreBufs b{};
    b.geo = (const grc::Geo *)ctx->geo_dev.p;
    b.rot_cs = (const double2 *)ctx->rot_cs.p;
    b.hkl = (const double *)ctx->hkl.p;
    b.vpos = (const double *)ctx->pos.p;
    b.U = (const double *)ctx->U.p;
    b.codes = ctx->mc.codes;
    b.codes8 = ctx->mc.codes8;
    b.vals = ctx->mc.vals;
    b.refine_list = (int64_t *)ctx->rlist.p;
    b.res = (grc::TrialRes *)ctx->res.p;
    b.work_counter = (int *)ctx->counter.p;
    b.bits = ctx->bits_ok ? (const uint32_t *)ctx->bits.p : nullptr;
    b.plane_words = ctx->plane_words;
    return b;
}

int stage_geo(grc_ctx *ctx) {
    TRY(ensure(ctx, ctx->geo_dev, sizeof(grc::Geo)));
    // unchanged since the last upload (byte for byte): the device copy is current, and the
    // kernels of this call are ordered after that upload on the same stream
    if (ctx->geo_up_ok && std::memcmp(&ctx->geo_up, &ctx->geo, sizeof(grc::Geo)) == 0) return GRC_OK;
    CU(cudaStreamSynchronize(ctx->stream));  // the pinned staging copy may still be read by an earlier call
    *ctx->geo_pinned = ctx->geo;
    CU(cudaMemcpyAsync(ctx->geo_dev.p, ctx->geo_pinned, sizeof(grc::Geo), cudaMemcpyHostToDevice, ctx->stream));
    std::memcpy(&ctx->geo_up, &ctx->geo, sizeof(grc::Geo));
    ctx->geo_up_ok = true;
    return GRC_OK;
}

// Scores n_trials trials into ctx->res.  comp: completeness only (no median; the packed hit mask).
// gkey (optional): first-maximum keys of every group of gsize consecutive trials, zeroed here.
int run_score(grc_ctx *ctx, const grc::Work &w, int64_t n_trials, bool comp = false,
              unsigned long long *gkey = nullptr, int64_t gsize = 0) {
    TRY(ensure(ctx, ctx->counter, 8 * sizeof(int)));
    TRY(stage_geo(ctx));
    if (comp) TRY(ensure_bits(ctx));
    if (gkey) CU(cudaMemsetAsync(gkey, 0, sizeof(unsigned long long) * ((n_trials + gsize - 1) / gsize), ctx->stream));
    int launches = 0;
    cudaEvent_t e0 = ctx->timing ? ctx->ev0 : nullptr, e1 = ctx->timing ? ctx->ev1 : nullptr;
    const int64_t round = ctx->force_path == 1 ? 0 : grc::sweep_round_trials(ctx->geo, ctx->num_sms);
    cudaError_t e;
    // Scan lists whose voxels carry at least a tile of orientations (a sweep tile then meets at
    // most two voxels) go to the sweep from 1/16 of a round: a one-voxel scan of 2,048
    // orientations already takes 0.27 ms there against 0.36 ms on the per-trial kernel (8,192:
    // 0.65 against 1.48 ms), while 1,024 favour the per-trial kernel.  Lists with a voxel per
    // trial or a few (grow rows, compete, trial lists) keep the half-round rule: there the two
    // kernels are within 3% of each other up to 16,384 trials.
    const bool shared_voxels = !w.items && !w.trial_voxel && !w.diag && w.n_or >= 64;
    const int64_t from = shared_voxels ? (round + 15) / 16 : (round + 1) / 2;
    bool fused_key = false;
    if (round > 0 && (ctx->force_path >= 2 || n_trials >= from)) {
        // projection-window scans (L2-resident map windows) for large trial counts: the warp scan,
        // or the CTA sweep when asked for by grc_set_path(2)
        TRY(ensure(ctx, ctx->rlist, sizeof(int64_t) * n_trials));
        grc::ScoreBufs b = bufs(ctx);
        if (comp && gkey) {  // completeness mode folds the first maximum per group in
            b.group_key = gkey;
            b.group_size = gsize;
            fused_key = true;
        }
        const int mode = comp ? grc::kScanComp : grc::kScanFull;
        // Full output over more than two scan rounds goes to the CTA sweep: its CTAs walk each
        // projection window in step and share the gathered 8-bit codes in L2 (FCC Al 2048^2 x 361,
        // 64 seeds x 32,768 orientations per call: 16.1 M trials/s against 13.5 M on the warp
        // scan).  Completeness-only calls and calls of one or two rounds take the warp scan (one
        // seed, full output: 15.9 against 15.3 M trials/s end to end; 64 seeds, completeness
        // only: 19.7 against 17.4 M).
        const bool sweep = ctx->force_path == 2 ||
                           (ctx->force_path == 0 && !comp &&
                            n_trials > 2 * grc::scan_round_trials(ctx->geo, ctx->num_sms));
        if (sweep) {
            e = grc::launch_sweep(ctx->geo, b, w, n_trials, ctx->num_sms, ctx->stream, e0, e1, &launches, 0, mode);
            ctx->stats.path = 2;
        } else {
            e = grc::launch_scan(ctx->geo, b, w, n_trials, ctx->num_sms, mode, ctx->stream, e0, e1, &launches);
            ctx->stats.path = 3;
        }
    } else {
        e = grc::launch_score(ctx->geo, bufs(ctx), w, ctx->num_sms, ctx->stream, e0, e1, &launches);
        ctx->stats.path = 1;
    }
    if (e != cudaSuccess) return fail(ctx, GRC_ECUDA, "scorer launch: %s", cudaGetErrorString(e));
    if (gkey && !fused_key) {
        CU(grc::launch_group_argmax((const grc::TrialRes *)ctx->res.p, n_trials, gsize, gkey, ctx->stream));
        ++launches;
    }
    ctx->timed_last = ctx->timing;
    ctx->stats.trials = n_trials;
    ctx->stats.kernel_launches += launches;
    return GRC_OK;
}

// First maximum per group from the keys of run_score into best/best_c (either may be NULL).
int decode_groups(grc_ctx *ctx, int64_t n_groups, int32_t *best, float *best_c) {
    if (!best && !best_c) return GRC_OK;
    CU(grc::launch_group_decode((const unsigned long long *)ctx->gkey.p, n_groups, best, best_c, ctx->stream));
    ++ctx->stats.kernel_launches;
    return GRC_OK;
}

// Seeding batch on device buffers: n_vox voxels x n_q orientations.  d_out (4 floats per trial)
// may be NULL when only the first maximum per voxel (best, best_c) is wanted.
int forward_device(grc_ctx *ctx, const float *d_pos, int64_t n_vox, const float *d_q, int64_t n_q, float *d_out,
                   int32_t *best = nullptr, float *best_c = nullptr) {
    TRY(check_ready(ctx));
    ctx->stats = grc_stats{};
    if (n_vox <= 0 || n_q <= 0) return GRC_OK;
    TRY(ensure(ctx, ctx->U, sizeof(double) * 9 * n_q));
    TRY(ensure(ctx, ctx->pos, sizeof(double) * 3 * n_vox));
    TRY(ensure(ctx, ctx->res, sizeof(grc::TrialRes) * n_vox * n_q));
    CU(grc::launch_quat_to_u(d_q, n_q, (double *)ctx->U.p, ctx->stream));
    CU(grc::launch_pos_f3(d_pos, n_vox, (double *)ctx->pos.p, ctx->stream));
    grc::Work w{};
    w.n_or = n_q;
    // Small calls (the per-trial kernel's range) get one work item per trial until every
    // resident CTA has one: an item's trials run one after another in one CTA.  Larger calls
    // keep kSeedChunk orientations per item, which shares the item's omega table among them.
    const int64_t fill = (int64_t)ctx->num_sms * 4;
    const int64_t chunk = std::max<int64_t>(1, std::min<int64_t>(kSeedChunk, n_vox * n_q / fill));
    w.chunk = (int32_t)chunk;
    w.chunks_per_voxel = (n_q + chunk - 1) / chunk;
    w.n_items = n_vox * w.chunks_per_voxel;
    const bool want_best = best || best_c;
    if (want_best) TRY(ensure(ctx, ctx->gkey, sizeof(unsigned long long) * n_vox));
    TRY(run_score(ctx, w, n_vox * n_q, !ctx->median, want_best ? (unsigned long long *)ctx->gkey.p : nullptr,
                  n_q));
    if (d_out) {
        CU(grc::launch_epi_forward((const grc::TrialRes *)ctx->res.p, n_vox * n_q, d_out, ctx->median,
                                   ctx->stream));
        ++ctx->stats.kernel_launches;
    }
    if (want_best) TRY(decode_groups(ctx, n_vox, best, best_c));
    ctx->stats.kernel_launches += 2;
    return GRC_OK;
}

int grow_device(grc_ctx *ctx, const float *d_rows6, int64_t m, const float *U9, const float *param1,
                float *d_out) {
    TRY(check_ready(ctx));
    ctx->stats = grc_stats{};
    if (!U9 || !param1) return fail(ctx, GRC_EINVAL, "grow: NULL U or param1");
    if (m <= 0) return GRC_OK;
    double p1[14];
    for (int i = 0; i < 14; ++i) {
        if (!std::isfinite(param1[i])) return fail(ctx, GRC_EINVAL, "param1(%d) is not finite", i + 1);
        p1[i] = param1[i];
    }
    TRY(ensure(ctx, ctx->p1, sizeof(p1)));
    TRY(ensure(ctx, ctx->in3, sizeof(float) * 9));
    TRY(ensure(ctx, ctx->U, sizeof(double) * 9));
    TRY(ensure(ctx, ctx->pos, sizeof(double) * 3 * m));
    TRY(ensure(ctx, ctx->res, sizeof(grc::TrialRes) * m));
    CU(cudaMemcpyAsync(ctx->p1.p, p1, sizeof(p1), cudaMemcpyHostToDevice, ctx->stream));
    CU(cudaMemcpyAsync(ctx->in3.p, U9, sizeof(float) * 9, cudaMemcpyHostToDevice, ctx->stream));
    CU(grc::launch_f9_to_u((const float *)ctx->in3.p, 1, (double *)ctx->U.p, ctx->stream));
    CU(grc::launch_pos_rows(d_rows6, 6, m, (const double *)ctx->p1.p, (double *)ctx->pos.p, ctx->stream));
    grc::Work w{};
    w.n_or = 1;
    w.chunk = 1;
    w.chunks_per_voxel = 1;
    w.n_items = m;
    TRY(run_score(ctx, w, m));
    CU(grc::launch_epi_grow((const grc::TrialRes *)ctx->res.p, d_rows6, m, (const double *)ctx->p1.p, d_out,
                            ctx->stream));
    ctx->stats.kernel_launches += 3;
    return GRC_OK;
}

int compete_device(grc_ctx *ctx, const float *d_rows5, int64_t m, const float *d_id, int64_t n_neigb,
                   const float *d_euler, int64_t n_grain, const float *param1, float *d_out, float *d_trial_out) {
    TRY(check_ready(ctx));
    ctx->stats = grc_stats{};
    if (!param1) return fail(ctx, GRC_EINVAL, "compete: NULL param1");
    if (m <= 0) return GRC_OK;
    if (n_grain < 1 || n_grain > (int64_t)INT32_MAX) return fail(ctx, GRC_EINVAL, "compete: bad grain count");
    double p1[14] = {0};
    for (int i = 0; i < 11; ++i) {
        if (!std::isfinite(param1[i])) return fail(ctx, GRC_EINVAL, "param1(%d) is not finite", i + 1);
        p1[i] = param1[i];
    }
    TRY(ensure(ctx, ctx->p1, sizeof(p1)));
    TRY(ensure(ctx, ctx->U, sizeof(double) * 9 * n_grain));
    TRY(ensure(ctx, ctx->pos, sizeof(double) * 3 * m));
    TRY(ensure(ctx, ctx->counts, sizeof(int64_t) * m));
    TRY(ensure(ctx, ctx->offsets, sizeof(int64_t) * m));
    TRY(ensure(ctx, ctx->items, sizeof(longlong4) * m));
    TRY(ensure(ctx, ctx->bad, sizeof(int)));
    CU(cudaMemcpyAsync(ctx->p1.p, p1, sizeof(p1), cudaMemcpyHostToDevice, ctx->stream));
    CU(cudaMemsetAsync(ctx->bad.p, 0, sizeof(int), ctx->stream));
    CU(grc::launch_euler_to_u(d_euler, n_grain, (double *)ctx->U.p, ctx->stream));
    CU(grc::launch_pos_rows(d_rows5, 5, m, (const double *)ctx->p1.p, (double *)ctx->pos.p, ctx->stream));
    CU(grc::launch_csr_counts(d_rows5, m, (int64_t *)ctx->counts.p, ctx->stream));
    size_t tmp_bytes = 0;
    CU(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, (int64_t *)ctx->counts.p, (int64_t *)ctx->offsets.p, m,
                                     ctx->stream));
    TRY(ensure(ctx, ctx->tmp, tmp_bytes));
    CU(cub::DeviceScan::ExclusiveSum(ctx->tmp.p, tmp_bytes, (int64_t *)ctx->counts.p, (int64_t *)ctx->offsets.p,
                                     m, ctx->stream));
    int64_t last_off = 0, last_cnt = 0;
    CU(cudaMemcpyAsync(&last_off, (int64_t *)ctx->offsets.p + (m - 1), 8, cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaMemcpyAsync(&last_cnt, (int64_t *)ctx->counts.p + (m - 1), 8, cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    const int64_t T = last_off + last_cnt;
    TRY(ensure(ctx, ctx->torient, sizeof(int32_t) * (T > 0 ? T : 1)));
    TRY(ensure(ctx, ctx->tvoxel, sizeof(int32_t) * (T > 0 ? T : 1)));
    TRY(ensure(ctx, ctx->res, sizeof(grc::TrialRes) * (T > 0 ? T : 1)));
    CU(grc::launch_csr_fill(d_rows5, m, (const int64_t *)ctx->offsets.p, d_id, n_neigb, n_grain,
                            (longlong4 *)ctx->items.p, (int32_t *)ctx->torient.p, (int32_t *)ctx->tvoxel.p,
                            (int *)ctx->bad.p, ctx->stream));
    int hbad = 0;
    CU(cudaMemcpyAsync(&hbad, ctx->bad.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    if (hbad & 1) return fail(ctx, GRC_EINVAL, "compete: a [first,last] range lies outside id_neigb_all");
    if (hbad & 2) return fail(ctx, GRC_EINVAL, "compete: a grain id lies outside the Euler table");
    if (T > 0) {
        grc::Work w{};
        w.items = (const longlong4 *)ctx->items.p;
        w.trial_orient = (const int32_t *)ctx->torient.p;
        w.trial_voxel = (const int32_t *)ctx->tvoxel.p;
        w.n_items = m;
        TRY(run_score(ctx, w, T));
    }
    CU(grc::launch_epi_compete((const grc::TrialRes *)ctx->res.p, (const longlong4 *)ctx->items.p,
                               (const int32_t *)ctx->torient.p, m, d_euler, d_out, d_trial_out, ctx->stream));
    ctx->stats.kernel_launches += 5;
    return GRC_OK;
}

// Copy a host array into a workspace buffer (or use it directly when already on the device).
int stage_in(grc_ctx *ctx, DevBuf &b, const float *src, int64_t n, const float **dst) {
    if (n <= 0) {
        *dst = nullptr;
        TRY(ensure(ctx, b, 16));
        *dst = (const float *)b.p;
        return GRC_OK;
    }
    if (!src) return fail(ctx, GRC_EINVAL, "NULL input array");
    if (is_device_ptr(src)) {
        *dst = src;
        return GRC_OK;
    }
    TRY(ensure(ctx, b, sizeof(float) * n));
    CU(cudaMemcpyAsync(b.p, src, sizeof(float) * n, cudaMemcpyHostToDevice, ctx->stream));
    *dst = (const float *)b.p;
    return GRC_OK;
}

struct Lock {
    grc_ctx *c;
    std::lock_guard<std::mutex> g;
    explicit Lock(grc_ctx *ctx) : c(ctx), g(ctx->mu) { cudaSetDevice(ctx->device); }
};

}  // namespace

extern "C" {

int grc_ctx_create(grc_ctx **out, int device) {
    if (!out) return GRC_EINVAL;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return GRC_ECUDA;
    }
    if (device < 0 || device >= n) return GRC_EINVAL;
    grc_ctx *ctx = new grc_ctx();
    ctx->device = device;
    cudaSetDevice(device);
    cudaDeviceProp p;
    if (cudaGetDeviceProperties(&p, device) != cudaSuccess) {
        delete ctx;
        return GRC_ECUDA;
    }
    if (p.major < 10) {
        delete ctx;
        return GRC_ECUDA;  // built for sm_100a only
    }
    ctx->num_sms = p.multiProcessorCount;
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaHostAlloc((void **)&ctx->geo_pinned, sizeof(grc::Geo), cudaHostAllocDefault) != cudaSuccess ||
        cudaEventCreate(&ctx->ev0) != cudaSuccess || cudaEventCreate(&ctx->ev1) != cudaSuccess) {
        delete ctx;
        return GRC_ECUDA;
    }
    *out = ctx;
    return GRC_OK;
}

int grc_ctx_destroy(grc_ctx *ctx) {
    if (!ctx) return GRC_EINVAL;
    {
        Lock l(ctx);
        cudaStreamSynchronize(ctx->stream);
        cudaFreeHost(ctx->geo_pinned);
        if (ctx->nm_active) cudaFreeHost(ctx->nm_active);
        DevBuf *all[] = {&ctx->nm, &ctx->sp_keys, &ctx->sp_ids, &ctx->sp_keys2, &ctx->sp_ids2, &ctx->cell_cnt, &ctx->cell_off, &ctx->pr_raw, &ctx->pr_keys, &ctx->pr_keys2, &ctx->pr_ids, &ctx->pr_ids2, &ctx->pcount, &ctx->fgeo, &ctx->fne, &ctx->ftrial, &ctx->fcost0, &ctx->fcost1, &ctx->fimp, &ctx->fhw,
                         &ctx->tvoxel, &ctx->rlist, &ctx->geo_dev, &ctx->rot_cs, &ctx->hkl, &ctx->pos, &ctx->U, &ctx->res, &ctx->in1, &ctx->in2,
                         &ctx->in3, &ctx->out, &ctx->items, &ctx->torient, &ctx->counts, &ctx->offsets,
                         &ctx->tmp, &ctx->counter, &ctx->p1, &ctx->bad, &ctx->bits, &ctx->gkey,
                         &ctx->sgrid, &ctx->sgrid32, &ctx->stv, &ctx->sto, &ctx->sbest, &ctx->nmloop};
        for (DevBuf *b : all) cudaFree(b->p);
        if (ctx->has_masks) {
            cudaFree(ctx->mc.codes);
            cudaFree(ctx->mc.codes8);
            cudaFree(ctx->mc.vals);
        }
        cudaEventDestroy(ctx->ev0);
        cudaEventDestroy(ctx->ev1);
        cudaStreamDestroy(ctx->stream);
    }
    delete ctx;
    return GRC_OK;
}

const char *grc_last_error(const grc_ctx *ctx) { return ctx ? ctx->err.c_str() : "NULL context"; }

void *grc_ctx_stream(grc_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

int grc_sync(grc_ctx *ctx) {
    if (!ctx) return GRC_EINVAL;
    Lock l(ctx);
    CU(cudaStreamSynchronize(ctx->stream));
    return GRC_OK;
}

int grc_set_options(grc_ctx *ctx, double dety0, double detz0, double thr) {
    if (!ctx) return GRC_EINVAL;
    Lock l(ctx);
    ctx->opt_dety0 = dety0;
    ctx->opt_detz0 = detz0;
    ctx->opt_thr = std::isnan(thr) ? 0.5 : thr;
    if (ctx->has_geo) apply_options(ctx);
    return GRC_OK;
}

int grc_upload_masks(grc_ctx *ctx, const float *map, int64_t dz, int64_t dy, int64_t nrot) {
    if (!ctx) return GRC_EINVAL;
    Lock l(ctx);
    if (map && is_device_ptr(map)) return upload_device_map(ctx, map, dz, dy, nrot);
    return upload_host_map(ctx, map, dz, dy, nrot);
}

int grc_upload_masks_device(grc_ctx *ctx, const float *d_map, int64_t dz, int64_t dy, int64_t nrot) {
    if (!ctx) return GRC_EINVAL;
    Lock l(ctx);
    if (!d_map) return fail(ctx, GRC_EINVAL, "proj_bin_bw is NULL");
    if (dz < 1 || dy < 1 || nrot < 1) return fail(ctx, GRC_EINVAL, "distance-map dimensions must be positive");
    return upload_device_map(ctx, d_map, dz, dy, nrot);
}

int grc_set_geometry(grc_ctx *ctx, const float *S, const float *B, const float *hkl, const float *rot,
                     const float *R, const float *param) {
    if (!ctx) return GRC_EINVAL;
    Lock l(ctx);
    return set_geometry(ctx, S, B, hkl, rot, R, param);
}

int grc_forward_comp(grc_ctx *ctx, const float *pos, const float *q, int64_t n_q, const float *S, const float *B,
                     const float *hkl, const float *map, const float *rot, const float *R, const float *param,
                     float *out) {
    if (!ctx) return GRC_EINVAL;
    Lock l(ctx);
    if (!pos || !out || (n_q > 0 && !q)) return fail(ctx, GRC_EINVAL, "forward_comp: NULL argument");
    if (n_q < 0) return fail(ctx, GRC_EINVAL, "forward_comp: negative orientation count");
    TRY(set_geometry(ctx, S, B, hkl, rot, R, param));
    if (map) TRY(upload_host_map(ctx, map, ctx->geo.detzsize, ctx->geo.detysize, ctx->geo.nrot));
    TRY(check_ready(ctx));
    if (n_q == 0) return GRC_OK;
    const float *d_pos = nullptr, *d_q = nullptr;
    TRY(stage_in(ctx, ctx->in1, pos, 3, &d_pos));
    TRY(stage_in(ctx, ctx->in2, q, 4 * n_q, &d_q));
    const bool dev_out = is_device_ptr(out);
    float *d_out = out;
    if (!dev_out) {
        TRY(ensure(ctx, ctx->out, sizeof(float) * 4 * n_q));
        d_out = (float *)ctx->out.p;
    }
    TRY(forward_device(ctx, d_pos, 1, d_q, n_q, d_out));
    if (!dev_out) CU(cudaMemcpyAsync(out, d_out, sizeof(float) * 4 * n_q, cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    CU(cudaGetLastError());
    return GRC_OK;
}

namespace {

// grc_grow_indexed_region with the context lock already held by the caller.
int grow_indexed_region_held(grc_ctx *ctx, const float *rows6, int64_t m, const float *U, const float *S,
                             const float *B, const float *hkl, const float *map, const float *rot, const float *R,
                             const float *param, const float *param1, float *out) {
    if (!U || !param1 || !out || (m > 0 && !rows6)) return fail(ctx, GRC_EINVAL, "grow: NULL argument");
    if (m < 0) return fail(ctx, GRC_EINVAL, "grow: negative row count");
    TRY(set_geometry(ctx, S, B, hkl, rot, R, param));
    if (map) TRY(upload_host_map(ctx, map, ctx->geo.detzsize, ctx->geo.detysize, ctx->geo.nrot));
    TRY(check_ready(ctx));
    if (m == 0) return GRC_OK;
    const float *d_rows = nullptr;
    TRY(stage_in(ctx, ctx->in1, rows6, 6 * m, &d_rows));
    const bool dev_out = is_device_ptr(out);
    float *d_out = out;
    if (!dev_out) {
        TRY(ensure(ctx, ctx->out, sizeof(float) * 7 * m));
        d_out = (float *)ctx->out.p;
    }
    TRY(grow_device(ctx, d_rows, m, U, param1, d_out));
    if (!dev_out) CU(cudaMemcpyAsync(out, d_out, sizeof(float) * 7 * m, cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    CU(cudaGetLastError());
    return GRC_OK;
}

}  // namespace

int grc_grow_indexed_region(grc_ctx *ctx, const float *rows6, int64_t m, const float *U, const float *S,
                            const float *B, const float *hkl, const float *map, const float *rot, const float *R,
                            const float *param, const float *param1, float *out) {
    if (!ctx) return GRC_EINVAL;
    Lock l(ctx);
    return grow_indexed_region_held(ctx, rows6, m, U, S, B, hkl, map, rot, R, param, param1, out);
}

namespace {

// Per-voxel score cache of a best-first walk for one orientation.  A request with unscored
// voxels scores, in one grc_grow_indexed_region call, every unscored in-mask voxel of the box
// that reaches kWalkHalo voxels beyond the unscored ones (and those themselves): the walk then
// makes one GPU call per few thousand voxels instead of one per step, with the same values.
constexpr int64_t kWalkHalo = 6;

struct WalkCache {
    grc_ctx *ctx;
    int64_t X, Y, Z;
    const double *mask;
    const float *U, *S, *B, *hkl, *map, *rot, *R, *param, *param1;
    std::vector<uint8_t> have;  // 0 unscored, 1 scored, 2 queued for this call
    std::vector<float> val;     // 3 per voxel: Nr_simu Nr_intersect dis_median
    std::vector<int32_t> todo;
    std::vector<float> rows, out;

    int64_t lin(int64_t x, int64_t y, int64_t z) const { return (x - 1) + X * ((y - 1) + Y * (z - 1)); }

    static int score(void *user, const int32_t *vox, int64_t n, double *res) {
        WalkCache &c = *static_cast<WalkCache *>(user);
        int64_t lo[3] = {INT64_MAX, INT64_MAX, INT64_MAX}, hi[3] = {0, 0, 0};
        bool miss = false;
        for (int64_t j = 0; j < n; ++j) {
            if (c.have[c.lin(vox[3 * j], vox[3 * j + 1], vox[3 * j + 2])]) continue;
            miss = true;
            for (int d = 0; d < 3; ++d) {
                lo[d] = std::min<int64_t>(lo[d], vox[3 * j + d]);
                hi[d] = std::max<int64_t>(hi[d], vox[3 * j + d]);
            }
        }
        if (miss) {
            const int64_t dims[3] = {c.X, c.Y, c.Z};
            for (int d = 0; d < 3; ++d) {
                lo[d] = std::max<int64_t>(lo[d] - kWalkHalo, 1);
                hi[d] = std::min<int64_t>(hi[d] + kWalkHalo, dims[d]);
            }
            c.todo.clear();
            auto queue = [&](int64_t x, int64_t y, int64_t z) {
                c.have[c.lin(x, y, z)] = 2;
                c.todo.push_back((int32_t)x);
                c.todo.push_back((int32_t)y);
                c.todo.push_back((int32_t)z);
            };
            for (int64_t z = lo[2]; z <= hi[2]; ++z)
                for (int64_t y = lo[1]; y <= hi[1]; ++y)
                    for (int64_t x = lo[0]; x <= hi[0]; ++x) {
                        const int64_t k = c.lin(x, y, z);
                        if (!c.have[k] && c.mask[k] > 0) queue(x, y, z);
                    }
            for (int64_t j = 0; j < n; ++j)  // requested voxels outside the mask too
                if (!c.have[c.lin(vox[3 * j], vox[3 * j + 1], vox[3 * j + 2])])
                    queue(vox[3 * j], vox[3 * j + 1], vox[3 * j + 2]);
            const int64_t m = (int64_t)c.todo.size() / 3;
            c.rows.assign(6 * m, 0.f);
            c.out.resize(7 * m);
            for (int64_t i = 0; i < m; ++i)
                for (int d = 0; d < 3; ++d) c.rows[6 * i + d] = (float)c.todo[3 * i + d];
            const int rc = grow_indexed_region_held(c.ctx, c.rows.data(), m, c.U, c.S, c.B, c.hkl, c.map, c.rot,
                                                    c.R, c.param, c.param1, c.out.data());
            if (rc != GRC_OK) return rc;
            c.map = nullptr;  // resident after the first call
            for (int64_t i = 0; i < m; ++i) {
                const int64_t k = c.lin(c.todo[3 * i], c.todo[3 * i + 1], c.todo[3 * i + 2]);
                for (int d = 0; d < 3; ++d) c.val[3 * k + d] = c.out[7 * i + 3 + d];
                c.have[k] = 1;
            }
        }
        for (int64_t j = 0; j < n; ++j) {
            const int64_t k = c.lin(vox[3 * j], vox[3 * j + 1], vox[3 * j + 2]);
            for (int d = 0; d < 3; ++d) res[3 * j + d] = (double)c.val[3 * k + d];
        }
        return GRC_OK;
    }
};

}  // namespace

int grc_grow_best_first(grc_ctx *ctx, int64_t X, int64_t Y, int64_t Z, const double *I, const double *Imask,
                        const double *DisMedian, const double *Ninter, const int32_t seed[3], double drop_off,
                        double maxD, double indexed_comp, double maxDmedian, const float *U, const float *S,
                        const float *B, const float *hkl, const float *map, const float *rot, const float *R,
                        const float *param, const float *param1, double *C_out, double *D_out, double *N_out,
                        uint8_t *J_out, int64_t *idx_out, int64_t idx_cap, int64_t *n_idx, double center[3],
                        int *replace_center) {
    if (!ctx) return GRC_EINVAL;
    // the lock is held for the whole walk, so the geometry and map its cached scores come from
    // cannot change between two blocks of scores
    Lock l(ctx);
    if (!I || !Imask || !DisMedian || !Ninter || !seed || !U || !param1 || !C_out || !D_out || !N_out || !J_out ||
        !n_idx || !center || !replace_center || (idx_cap > 0 && !idx_out))
        return fail(ctx, GRC_EINVAL, "grow_best_first: NULL argument");
    if (X < 1 || Y < 1 || Z < 1 || X > INT32_MAX || Y > INT32_MAX || Z > INT32_MAX || X * Y > INT64_MAX / Z)
        return fail(ctx, GRC_EINVAL, "grow_best_first: bad volume size");
    if (seed[0] < 1 || seed[1] < 1 || seed[2] < 1 || seed[0] > X || seed[1] > Y || seed[2] > Z)
        return fail(ctx, GRC_EINVAL, "grow_best_first: seed outside the volume");
    // only the first 11 floats of param1 place voxels; the grow kernel's own thresholds
    // (seed_comp, drop_off, maxDmedian) are not used by the walk and may hold anything
    float p1[14];
    for (int i = 0; i < 14; ++i) p1[i] = i < 11 ? param1[i] : 0.f;
    WalkCache c{ctx, X, Y, Z, Imask, U, S, B, hkl, map, rot, R, param, p1};
    c.have.assign((size_t)(X * Y * Z), 0);
    c.val.assign((size_t)(3 * X * Y * Z), 0.f);
    const int rc = grc_walk_best_first(&WalkCache::score, &c, X, Y, Z, I, Imask, DisMedian, Ninter, seed, drop_off,
                                       maxD, indexed_comp, maxDmedian, C_out, D_out, N_out, J_out, idx_out, idx_cap,
                                       n_idx, center, replace_center);
    if (rc == GRC_ECAPACITY) return fail(ctx, GRC_ECAPACITY, "grow_best_first: more grown voxels than idx_cap");
    return rc;  // arguments were checked above: any other error is the scorer's, recorded by the grow scorer
}

int grc_forward_comp_compete(grc_ctx *ctx, const float *rows5, int64_t m, const float *id_neigb, int64_t n_neigb,
                             const float *euler, int64_t n_grain, const float *S, const float *B, const float *hkl,
                             const float *map, const float *rot, const float *R, const float *param,
                             const float *param1, float *out) {
    if (!ctx) return GRC_EINVAL;
    Lock l(ctx);
    if (!param1 || !out || (m > 0 && (!rows5 || !euler))) return fail(ctx, GRC_EINVAL, "compete: NULL argument");
    if (m < 0 || n_neigb < 0 || n_grain < 0) return fail(ctx, GRC_EINVAL, "compete: negative size");
    TRY(set_geometry(ctx, S, B, hkl, rot, R, param));
    if (map) TRY(upload_host_map(ctx, map, ctx->geo.detzsize, ctx->geo.detysize, ctx->geo.nrot));
    TRY(check_ready(ctx));
    if (m == 0) return GRC_OK;
    const float *d_rows = nullptr, *d_id = nullptr, *d_eu = nullptr;
    TRY(stage_in(ctx, ctx->in1, rows5, 5 * m, &d_rows));
    TRY(stage_in(ctx, ctx->in2, id_neigb, n_neigb, &d_id));
    TRY(stage_in(ctx, ctx->in3, euler, 3 * n_grain, &d_eu));
    const bool dev_out = is_device_ptr(out);
    float *d_out = out;
    if (!dev_out) {
        TRY(ensure(ctx, ctx->out, sizeof(float) * 8 * m));
        d_out = (float *)ctx->out.p;
    }
    TRY(compete_device(ctx, d_rows, m, d_id, n_neigb, d_eu, n_grain, param1, d_out, nullptr));
    if (!dev_out) CU(cudaMemcpyAsync(out, d_out, sizeof(float) * 8 * m, cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    CU(cudaGetLastError());
    return GRC_OK;
}

int grc_forward_comp_device(grc_ctx *ctx, const float *d_pos, int64_t n_vox, const float *d_q, int64_t n_q,
                            float *d_out) {
    if (!ctx) return GRC_EINVAL;
    Lock l(ctx);
    if (n_vox < 0 || n_q < 0) return fail(ctx, GRC_EINVAL, "negative size");
    if (n_vox > 0 && n_q > 0 && (!d_pos || !d_q || !d_out)) return fail(ctx, GRC_EINVAL, "NULL device buffer");
    if (n_vox > 0 && n_q > 0) {
        TRY(need_device(ctx, d_pos, "d_pos"));
        TRY(need_device(ctx, d_q, "d_q"));
        TRY(need_device(ctx, d_out, "d_out"));
    }
    return forward_device(ctx, d_pos, n_vox, d_q, n_q, d_out);
}

int grc_grow_device(grc_ctx *ctx, const float *d_rows6, int64_t m, const float *U, const float *param1,
                    float *d_out) {
    if (!ctx) return GRC_EINVAL;
    Lock l(ctx);
    if (m < 0) return fail(ctx, GRC_EINVAL, "negative size");
    if (m > 0 && (!d_rows6 || !d_out)) return fail(ctx, GRC_EINVAL, "NULL device buffer");
    if (m > 0) {
        TRY(need_device(ctx, d_rows6, "d_rows6"));
        TRY(need_device(ctx, d_out, "d_out"));
    }
    return grow_device(ctx, d_rows6, m, U, param1, d_out);
}

int grc_compete_device(grc_ctx *ctx, const float *d_rows5, int64_t m, const float *d_id, int64_t n_neigb,
                       const float *d_euler, int64_t n_grain, const float *param1, float *d_out,
                       float *d_trial_out) {
    if (!ctx) return GRC_EINVAL;
    Lock l(ctx);
    if (m < 0 || n_neigb < 0 || n_grain < 0) return fail(ctx, GRC_EINVAL, "negative size");
    if (m > 0 && (!d_rows5 || !d_out || !d_euler)) return fail(ctx, GRC_EINVAL, "NULL device buffer");
    if (m > 0) {
        TRY(need_device(ctx, d_rows5, "d_rows5"));
        TRY(need_device(ctx, d_id, "d_id_neigb"));
        TRY(need_device(ctx, d_euler, "d_euler"));
        TRY(need_device(ctx, d_out, "d_out"));
        TRY(need_device(ctx, d_trial_out, "d_trial_out"));
    }
    return compete_device(ctx, d_rows5, m, d_id, n_neigb, d_euler, n_grain, param1, d_out, d_trial_out);
}

}  // extern "C"

namespace {

// grc_score_trials_device and its argmax form (context lock held).  d_out may be NULL when
// group_size > 0 (first maximum per group only).
int score_trials(grc_ctx *ctx, const double *d_pos, int64_t n_vox, const double *d_q, int64_t n_q,
                 const int32_t *d_tv, const int32_t *d_to, int64_t n_trials, float *d_out, int64_t group_size,
                 int32_t *best, float *best_c) {
    TRY(check_ready(ctx));
    ctx->stats = grc_stats{};
    if (n_trials < 0 || n_vox < 0 || n_q < 0) return fail(ctx, GRC_EINVAL, "negative size");
    if (group_size < 0 || (group_size > 0 && n_trials % group_size != 0))
        return fail(ctx, GRC_EINVAL, "trials: n_trials must be a multiple of group_size");
    if (n_trials == 0) return GRC_OK;
    if (!d_pos || !d_q || (!d_out && group_size == 0) || n_vox < 1 || n_q < 1)
        return fail(ctx, GRC_EINVAL, "trials: NULL buffer or no rows");
    TRY(need_device(ctx, best, "trials: d_best"));
    TRY(need_device(ctx, best_c, "trials: d_best_c"));
    TRY(need_device(ctx, d_pos, "trials: d_pos"));
    TRY(need_device(ctx, d_q, "trials: d_q"));
    TRY(need_device(ctx, d_out, "trials: d_out"));
    TRY(need_device(ctx, d_tv, "trials: d_trial_voxel"));
    TRY(need_device(ctx, d_to, "trials: d_trial_orient"));
    if ((d_tv == nullptr) != (d_to == nullptr))
        return fail(ctx, GRC_EINVAL, "trials: give both index arrays or neither");
    if (!d_tv && (n_vox != n_trials || n_q != n_trials))
        return fail(ctx, GRC_EINVAL, "trials: without index arrays n_vox and n_q must equal n_trials");
    if (n_vox > (int64_t)INT32_MAX || n_q > (int64_t)INT32_MAX)
        return fail(ctx, GRC_ECAPACITY, "trials: more than 2^31-1 voxels or orientations");
    TRY(ensure(ctx, ctx->U, sizeof(double) * 9 * n_q));
    TRY(ensure(ctx, ctx->pos, sizeof(double) * 3 * n_vox));
    TRY(ensure(ctx, ctx->res, sizeof(grc::TrialRes) * n_trials));
    CU(grc::launch_quat_to_u_d(d_q, n_q, (double *)ctx->U.p, ctx->stream));
    CU(cudaMemcpyAsync(ctx->pos.p, d_pos, sizeof(double) * 3 * n_vox, cudaMemcpyDeviceToDevice, ctx->stream));
    grc::Work w{};
    if (d_tv) {
        TRY(ensure(ctx, ctx->items, sizeof(longlong4) * n_trials));
        TRY(ensure(ctx, ctx->bad, 2 * sizeof(int)));
        CU(cudaMemsetAsync(ctx->bad.p, 0, 2 * sizeof(int), ctx->stream));
        CU(grc::launch_trial_items(d_tv, d_to, n_trials, n_vox, n_q, (longlong4 *)ctx->items.p, (int *)ctx->bad.p,
                                   ctx->stream));
        int hbad[2] = {0, 0};
        CU(cudaMemcpyAsync(hbad, ctx->bad.p, 2 * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
        CU(cudaStreamSynchronize(ctx->stream));
        if (hbad[0]) return fail(ctx, GRC_EINVAL, "trials: a voxel or orientation index lies out of range");
        w.starts_per_32 = hbad[1];
        w.items = (const longlong4 *)ctx->items.p;
        w.trial_orient = d_to;
        w.trial_voxel = d_tv;
        w.n_items = n_trials;
    } else {
        w.diag = 1;
        w.n_or = 1;
        w.chunk = 1;
        w.chunks_per_voxel = 1;
        w.n_items = n_trials;
    }
    const int64_t n_groups = group_size > 0 ? n_trials / group_size : 0;
    if (n_groups > 0) TRY(ensure(ctx, ctx->gkey, sizeof(unsigned long long) * n_groups));
    TRY(run_score(ctx, w, n_trials, !ctx->median, n_groups > 0 ? (unsigned long long *)ctx->gkey.p : nullptr,
                  group_size));
    if (d_out) {
        CU(grc::launch_epi_forward((const grc::TrialRes *)ctx->res.p, n_trials, d_out, ctx->median, ctx->stream));
        ++ctx->stats.kernel_launches;
    }
    if (n_groups > 0) TRY(decode_groups(ctx, n_groups, best, best_c));
    ctx->stats.kernel_launches += 2 + (d_tv ? 1 : 0);
    return GRC_OK;
}

}  // namespace

extern "C" {

int grc_score_trials_device(grc_ctx *ctx, const double *d_pos, int64_t n_vox, const double *d_q, int64_t n_q,
                            const int32_t *d_tv, const int32_t *d_to, int64_t n_trials, float *d_out) {
    if (!ctx) return GRC_EINVAL;
    Lock l(ctx);
    return score_trials(ctx, d_pos, n_vox, d_q, n_q, d_tv, d_to, n_trials, d_out, 0, nullptr, nullptr);
}

int grc_score_trials_argmax_device(grc_ctx *ctx, const double *d_pos, int64_t n_vox, const double *d_q, int64_t n_q,
                                   const int32_t *d_tv, const int32_t *d_to, int64_t n_trials, int64_t group_size,
                                   float *d_out, int32_t *d_best, float *d_best_c) {
    if (!ctx) return GRC_EINVAL;
    Lock l(ctx);
    if (group_size < 1) return fail(ctx, GRC_EINVAL, "trials: group_size must be positive");
    return score_trials(ctx, d_pos, n_vox, d_q, n_q, d_tv, d_to, n_trials, d_out, group_size, d_best, d_best_c);
}

int grc_forward_comp_argmax_device(grc_ctx *ctx, const float *d_pos, int64_t n_vox, const float *d_q, int64_t n_q,
                                   float *d_out, int32_t *d_best, float *d_best_c) {
    if (!ctx) return GRC_EINVAL;
    Lock l(ctx);
    if (n_vox < 0 || n_q < 0) return fail(ctx, GRC_EINVAL, "negative size");
    if (n_vox > 0 && n_q > 0) {
        if (!d_pos || !d_q) return fail(ctx, GRC_EINVAL, "NULL device buffer");
        TRY(need_device(ctx, d_pos, "d_pos"));
        TRY(need_device(ctx, d_q, "d_q"));
        TRY(need_device(ctx, d_out, "d_out"));
        TRY(need_device(ctx, d_best, "d_best"));
        TRY(need_device(ctx, d_best_c, "d_best_c"));
    }
    return forward_device(ctx, d_pos, n_vox, d_q, n_q, d_out, d_best, d_best_c);
}

int grc_seed_candidates_device(grc_ctx *ctx, const float *d_pos, int64_t n, const float *d_q, const double *d_q64,
                               int64_t n_q, int n_top, int32_t *d_idx, double *d_cand, float *d_out) {
    if (!ctx) return GRC_EINVAL;
    Lock l(ctx);
    if (n < 0 || n_q < 0) return fail(ctx, GRC_EINVAL, "seed candidates: negative size");
    if (n == 0) return GRC_OK;
    if (!d_pos || !d_q || !d_idx || n_q < 1) return fail(ctx, GRC_EINVAL, "seed candidates: NULL buffer");
    if (n_top < 1 || n_top > 4096 || n_top > n_q)
        return fail(ctx, GRC_EINVAL, "seed candidates: n_top must lie in 1..min(4096, n_q)");
    if (n > (int64_t)INT32_MAX || n_q > (int64_t)INT32_MAX) return fail(ctx, GRC_ECAPACITY, "seed candidates: too many rows");
    TRY(need_device(ctx, d_pos, "d_pos"));
    TRY(need_device(ctx, d_q, "d_q"));
    TRY(need_device(ctx, d_q64, "d_q64"));
    TRY(need_device(ctx, d_idx, "d_idx"));
    TRY(need_device(ctx, d_cand, "d_cand"));
    TRY(need_device(ctx, d_out, "d_out"));
    const bool med = ctx->median;
    ctx->median = false;  // the engine reads column 3 only
    const int rc = forward_device(ctx, d_pos, n, d_q, n_q, d_out);
    ctx->median = med;
    TRY(rc);
    CU(grc::launch_top_rows(nullptr, (const grc::TrialRes *)ctx->res.p, 1, n, n_q, n_top, d_idx, ctx->stream));
    int launches = 1;
    if (d_cand) {
        CU(grc::launch_gather_rows(d_idx, n, n_top, n_q, d_q64 ? nullptr : d_q, d_q64, 0, 4, d_cand, ctx->stream));
        ++launches;
    }
    ctx->stats.kernel_launches += launches;
    return GRC_OK;
}

int grc_seed_refine_device(grc_ctx *ctx, const double *d_pos, int64_t n, const double *d_cand, int k, int nr,
                           double gridsize, int n_x0, double *d_best_q, float *d_best_c, int32_t *d_order,
                           double *d_x0) {
    if (!ctx) return GRC_EINVAL;
    Lock l(ctx);
    if (n < 0 || k < 0) return fail(ctx, GRC_EINVAL, "seed refine: negative size");
    if (n == 0 || k == 0) return GRC_OK;
    if (!d_pos || !d_cand || !d_best_q || !d_best_c || !d_order) return fail(ctx, GRC_EINVAL, "seed refine: NULL buffer");
    if (nr < 0 || grc::local_grid_rows(nr) > 1024 || !(gridsize > 0))
        return fail(ctx, GRC_EINVAL, "seed refine: nr must give at most 1024 grid rows, gridsize > 0");
    if (k > 4096) return fail(ctx, GRC_EINVAL, "seed refine: at most 4096 candidates per seed");
    if (d_x0 && (n_x0 < 1 || n_x0 > k)) return fail(ctx, GRC_EINVAL, "seed refine: n_x0 must lie in 1..k");
    const int64_t L = grc::local_grid_rows(nr), n_cand = n * (int64_t)k, n_trials = n_cand * L;
    if (n_trials > (int64_t)INT32_MAX) return fail(ctx, GRC_ECAPACITY, "seed refine: more than 2^31-1 trials");
    TRY(need_device(ctx, d_pos, "d_pos"));
    TRY(need_device(ctx, d_cand, "d_cand"));
    TRY(need_device(ctx, d_best_q, "d_best_q"));
    TRY(need_device(ctx, d_best_c, "d_best_c"));
    TRY(need_device(ctx, d_order, "d_order"));
    TRY(need_device(ctx, d_x0, "d_x0"));
    TRY(ensure(ctx, ctx->sgrid, sizeof(double) * 4 * n_trials));
    TRY(ensure(ctx, ctx->sgrid32, sizeof(double) * 4 * n_trials));
    TRY(ensure(ctx, ctx->stv, sizeof(int32_t) * n_trials));
    TRY(ensure(ctx, ctx->sto, sizeof(int32_t) * n_trials));
    TRY(ensure(ctx, ctx->sbest, sizeof(int32_t) * n_cand + sizeof(float) * n_cand + sizeof(double) * 4 * n_cand));
    int32_t *gbest = (int32_t *)ctx->sbest.p;                                   // grid row of each maximum
    float *cbest = (float *)(gbest + n_cand);                                   // its completeness
    double *qbest = (double *)(((uintptr_t)(cbest + n_cand) + 15) & ~(uintptr_t)15);  // its FP64 grid row
    CU(grc::launch_local_grid(d_cand, n_cand, nr, gridsize, (double *)ctx->sgrid.p, (double *)ctx->sgrid32.p, nullptr,
                              ctx->stream));
    CU(grc::launch_block_lists(n_trials, (int64_t)k * L, (int32_t *)ctx->stv.p, (int32_t *)ctx->sto.p, ctx->stream));
    const bool med = ctx->median;
    ctx->median = false;  // fit_OR_constrain_with_local_comp_cuda.m:105 reads column 3 only
    const int rc = score_trials(ctx, d_pos, n, (const double *)ctx->sgrid32.p, n_trials, (const int32_t *)ctx->stv.p,
                                (const int32_t *)ctx->sto.p, n_trials, nullptr, L, gbest, cbest);
    ctx->median = med;
    TRY(rc);
    // each candidate's maximum as its FP64 grid row, then the candidates of every seed in
    // sortrows(Output_max, 3, 'descend') order (:112): rows, completeness, candidate index, x0
    CU(grc::launch_gather_rows(gbest, n_cand, 1, L, nullptr, (const double *)ctx->sgrid.p, L, 4, qbest, ctx->stream));
    CU(grc::launch_top_rows(cbest, nullptr, 1, n, k, k, d_order, ctx->stream));
    CU(grc::launch_gather_rows(d_order, n, k, k, nullptr, qbest, k, 4, d_best_q, ctx->stream));
    CU(grc::launch_gather_floats(d_order, n, k, k, cbest, k, d_best_c, ctx->stream));
    int launches = 6;
    if (d_x0) {
        CU(grc::launch_take_x0(d_best_q, n, k, n_x0, d_x0, ctx->stream));
        ++launches;
    }
    ctx->stats.kernel_launches += launches;
    return GRC_OK;
}

int grc_local_grid_device(grc_ctx *ctx, const double *d_cand, int64_t n_cand, int nr, double gridsize,
                          double *d_rows, float *d_rows_f32) {
    if (!ctx) return GRC_EINVAL;
    Lock l(ctx);
    if (n_cand < 0) return fail(ctx, GRC_EINVAL, "local grid: negative size");
    if (n_cand == 0) return GRC_OK;
    if (!d_cand || !d_rows) return fail(ctx, GRC_EINVAL, "local grid: NULL buffer");
    if (nr < 0 || grc::local_grid_rows(nr) > 1024 || !(gridsize > 0))
        return fail(ctx, GRC_EINVAL, "local grid: nr must give at most 1024 grid rows, gridsize > 0");
    TRY(need_device(ctx, d_cand, "d_cand"));
    TRY(need_device(ctx, d_rows, "d_rows"));
    TRY(need_device(ctx, d_rows_f32, "d_rows_f32"));
    CU(grc::launch_local_grid(d_cand, n_cand, nr, gridsize, d_rows, nullptr, d_rows_f32, ctx->stream));
    return GRC_OK;
}

uint64_t grc_map_key(const float *map, int64_t n, int64_t samples) {
    // FNV-1a over n and the bit patterns of the sampled values (every value when n <= samples)
    uint64_t h = 1469598103934665603ull;
    auto mix = [&](uint64_t v) {
        for (int b = 0; b < 8; ++b) {
            h ^= (v >> (8 * b)) & 0xffu;
            h *= 1099511628211ull;
        }
    };
    mix((uint64_t)n);
    if (!map || n <= 0) return h | 1;
    if (samples <= 0 || samples > n) samples = n;
    for (int64_t k = 0; k < samples; ++k) {
        const int64_t i = samples == n ? k : (int64_t)((__int128)k * (n - 1) / (samples - 1 > 0 ? samples - 1 : 1));
        uint32_t bits;
        std::memcpy(&bits, map + i, 4);
        mix(((uint64_t)i << 32) | bits);
    }
    return h | 1;  // never 0, the "no key" value
}

int grc_upload_masks_if_changed(grc_ctx *ctx, const float *map, int64_t detzsize, int64_t detysize, int64_t nrot,
                                int64_t samples, int *uploaded) {
    if (!ctx) return GRC_EINVAL;
    Lock l(ctx);
    if (uploaded) *uploaded = 0;
    if (!map) return fail(ctx, GRC_EINVAL, "proj_bin_bw is NULL");
    if (detzsize < 1 || detysize < 1 || nrot < 1) return fail(ctx, GRC_EINVAL, "distance-map dimensions must be positive");
    const uint64_t key = grc_map_key(map, detzsize * detysize * nrot, samples);
    if (ctx->has_masks && ctx->map_key == key && ctx->mz == detzsize && ctx->my == detysize && ctx->mrot == nrot)
        return GRC_OK;
    TRY(upload_host_map(ctx, map, detzsize, detysize, nrot));
    ctx->map_key = key;
    if (uploaded) *uploaded = 1;
    return GRC_OK;
}

}  // extern "C"

namespace {

// Distance map from binary spot images on the device: bwdist (exact EDT) of every projection, then
// the rank coding of upload_device_map.  d_mask: one byte per pixel (nonzero = spot).
int upload_spot_device(grc_ctx *ctx, const uint8_t *d_mask, int64_t dz, int64_t dy, int64_t nrot) {
    const int64_t n = dz * dy * nrot;
    float *d_map = nullptr;
    cudaError_t e = cudaMalloc(&d_map, sizeof(float) * n);
    if (e != cudaSuccess) return fail(ctx, GRC_ECUDA, "cudaMalloc(distance map): %s", cudaGetErrorString(e));
    e = grc::launch_edt(d_mask, dz, dy, nrot, d_map, ctx->stream);
    int r = e == cudaSuccess ? upload_device_map(ctx, d_map, dz, dy, nrot)
                             : fail(ctx, GRC_ECUDA, "bwdist: %s", cudaGetErrorString(e));
    cudaStreamSynchronize(ctx->stream);
    cudaFree(d_map);
    return r;
}

int upload_spot_host(grc_ctx *ctx, const uint8_t *mask, int64_t dz, int64_t dy, int64_t nrot) {
    const int64_t n = dz * dy * nrot;
    uint8_t *d_mask = nullptr;
    cudaError_t e = cudaMalloc(&d_mask, n);
    if (e != cudaSuccess) return fail(ctx, GRC_ECUDA, "cudaMalloc(spot masks): %s", cudaGetErrorString(e));
    e = cudaMemcpyAsync(d_mask, mask, n, cudaMemcpyHostToDevice, ctx->stream);
    int r = e == cudaSuccess ? upload_spot_device(ctx, d_mask, dz, dy, nrot)
                             : fail(ctx, GRC_ECUDA, "spot-mask upload: %s", cudaGetErrorString(e));
    cudaStreamSynchronize(ctx->stream);
    cudaFree(d_mask);
    return r;
}

// Packed-mask file: this header, then nrot * plane_words little-endian 32-bit words (bit p&31 of
// word p>>5 of each projection = spot pixel p, p = (dety-1)*detzsize + (detz-1)).
struct PackedHeader {
    char magic[8];          // "GRCMASK1"
    uint32_t version;       // 1
    uint32_t header_bytes;  // sizeof(PackedHeader)
    int64_t detzsize, detysize, nrot, plane_words;
    uint64_t key;           // FNV-1a of the words
    uint64_t reserved[3];
};
static_assert(sizeof(PackedHeader) == 80, "packed-mask header layout");
const char kPackedMagic[8] = {'G', 'R', 'C', 'M', 'A', 'S', 'K', '1'};

uint64_t words_key(const uint32_t *w, int64_t n) {
    uint64_t h = 1469598103934665603ull;
    for (int64_t i = 0; i < n; ++i) {
        uint32_t v = w[i];
        for (int b = 0; b < 4; ++b) {
            h ^= (v >> (8 * b)) & 0xffu;
            h *= 1099511628211ull;
        }
    }
    return h;
}

}  // namespace

extern "C" {

int grc_upload_spot_masks(grc_ctx *ctx, const uint8_t *proj_bin, int64_t detzsize, int64_t detysize, int64_t nrot) {
    if (!ctx) return GRC_EINVAL;
    Lock l(ctx);
    if (!proj_bin) return fail(ctx, GRC_EINVAL, "proj_bin is NULL");
    if (detzsize < 1 || detysize < 1 || nrot < 1) return fail(ctx, GRC_EINVAL, "spot-mask dimensions must be positive");
    if (is_device_ptr(proj_bin)) return upload_spot_device(ctx, proj_bin, detzsize, detysize, nrot);
    return upload_spot_host(ctx, proj_bin, detzsize, detysize, nrot);
}

int grc_save_packed_masks(grc_ctx *ctx, const char *path) {
    if (!ctx) return GRC_EINVAL;
    Lock l(ctx);
    if (!path) return fail(ctx, GRC_EINVAL, "save: NULL path");
    if (!ctx->has_masks) return fail(ctx, GRC_ENOMASK, "save: no map resident");
    const int64_t plane = ctx->mz * ctx->my, pw = (plane + 127) / 128 * 4, nw = pw * ctx->mrot;
    // spot pixels = distance 0 = code 0 when the smallest distinct value is 0
    const uint32_t n_spot = (!ctx->h_vals.empty() && ctx->h_vals[0] == 0.0f) ? 1u : 0u;
    uint32_t *d_bits = nullptr;
    cudaError_t e = cudaMalloc(&d_bits, sizeof(uint32_t) * nw);
    if (e != cudaSuccess) return fail(ctx, GRC_ECUDA, "save: cudaMalloc: %s", cudaGetErrorString(e));
    std::vector<uint32_t> h((size_t)nw);
    e = grc::launch_pack_bits(ctx->mc.codes8, 1, plane, ctx->mrot, n_spot, pw, d_bits, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), d_bits, sizeof(uint32_t) * nw, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    cudaFree(d_bits);
    if (e != cudaSuccess) return fail(ctx, GRC_ECUDA, "save: %s", cudaGetErrorString(e));
    PackedHeader hd{};
    std::memcpy(hd.magic, kPackedMagic, 8);
    hd.version = 1;
    hd.header_bytes = sizeof(PackedHeader);
    hd.detzsize = ctx->mz;
    hd.detysize = ctx->my;
    hd.nrot = ctx->mrot;
    hd.plane_words = pw;
    hd.key = words_key(h.data(), nw);
    FILE *f = std::fopen(path, "wb");
    if (!f) return fail(ctx, GRC_EINVAL, "save: cannot open %s", path);
    const bool ok = std::fwrite(&hd, sizeof hd, 1, f) == 1 &&
                    std::fwrite(h.data(), sizeof(uint32_t), (size_t)nw, f) == (size_t)nw;
    const bool closed = std::fclose(f) == 0;
    if (!ok || !closed) return fail(ctx, GRC_EINVAL, "save: write to %s failed", path);
    return GRC_OK;
}

int grc_load_packed_masks(grc_ctx *ctx, const char *path) {
    if (!ctx) return GRC_EINVAL;
    Lock l(ctx);
    if (!path) return fail(ctx, GRC_EINVAL, "load: NULL path");
    FILE *f = std::fopen(path, "rb");
    if (!f) return fail(ctx, GRC_EINVAL, "load: cannot open %s", path);
    PackedHeader hd{};
    if (std::fread(&hd, sizeof hd, 1, f) != 1 || std::memcmp(hd.magic, kPackedMagic, 8) != 0 || hd.version != 1 ||
        hd.header_bytes != sizeof(PackedHeader)) {
        std::fclose(f);
        return fail(ctx, GRC_EINVAL, "load: %s is not a packed-mask file (version 1)", path);
    }
    // the same limits as a map given to grc_upload_masks (set_geometry: 10^6 pixels per side,
    // 2^31 - 1 per projection), checked before anything is allocated
    if (hd.detzsize < 1 || hd.detysize < 1 || hd.nrot < 1 || hd.detzsize > 1000000 || hd.detysize > 1000000 ||
        hd.detzsize * hd.detysize > 2147483647LL || hd.nrot > GRC_MAX_NROT ||
        hd.plane_words != (hd.detzsize * hd.detysize + 127) / 128 * 4) {
        std::fclose(f);
        return fail(ctx, GRC_EINVAL, "load: %s has an inconsistent header", path);
    }
    const int64_t nw = hd.plane_words * hd.nrot, plane = hd.detzsize * hd.detysize;
    // the file must hold exactly the header and the words it announces
    const long here = std::ftell(f);
    const bool sized = here >= 0 && std::fseek(f, 0, SEEK_END) == 0 &&
                       (int64_t)std::ftell(f) == (int64_t)sizeof(PackedHeader) + 4 * nw &&
                       std::fseek(f, here, SEEK_SET) == 0;
    if (!sized) {
        std::fclose(f);
        return fail(ctx, GRC_EINVAL, "load: %s is truncated or longer than its header says", path);
    }
    std::vector<uint32_t> h;
    try {
        h.resize((size_t)nw);
    } catch (const std::bad_alloc &) {
        std::fclose(f);
        return fail(ctx, GRC_ECAPACITY, "load: %lld words do not fit in host memory", (long long)nw);
    }
    const bool full = std::fread(h.data(), sizeof(uint32_t), (size_t)nw, f) == (size_t)nw;
    std::fclose(f);
    if (!full) return fail(ctx, GRC_EINVAL, "load: %s is truncated", path);
    if (words_key(h.data(), nw) != hd.key) return fail(ctx, GRC_EINVAL, "load: %s fails its content key", path);
    uint32_t *d_bits = nullptr;
    uint8_t *d_mask = nullptr;
    cudaError_t e = cudaMalloc(&d_bits, sizeof(uint32_t) * nw);
    if (e == cudaSuccess) e = cudaMalloc(&d_mask, plane * hd.nrot);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_bits, h.data(), sizeof(uint32_t) * nw, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = grc::launch_unpack_bits(d_bits, plane, hd.nrot, hd.plane_words, d_mask, ctx->stream);
    int r = e == cudaSuccess ? upload_spot_device(ctx, d_mask, hd.detzsize, hd.detysize, hd.nrot)
                             : fail(ctx, GRC_ECUDA, "load: %s", cudaGetErrorString(e));
    cudaStreamSynchronize(ctx->stream);
    cudaFree(d_bits);
    cudaFree(d_mask);
    return r;
}

int grc_set_median(grc_ctx *ctx, int enable) {
    if (!ctx) return GRC_EINVAL;
    Lock l(ctx);
    ctx->median = enable != 0;
    return GRC_OK;
}

int grc_fit_orientation_nm(grc_ctx *ctx, const double *d_pos, const double *d_x0, int64_t n, double half_width,
                           int max_evals, int max_iter, double tol_f, double tol_x, double *d_x, double *d_fval,
                           int32_t *d_evals, int32_t *d_iters, int32_t *d_flag) {
    if (!ctx) return GRC_EINVAL;
    Lock l(ctx);
    TRY(check_ready(ctx));
    ctx->stats = grc_stats{};
    if (n < 0) return fail(ctx, GRC_EINVAL, "negative size");
    if (n == 0) return GRC_OK;
    if (!d_pos || !d_x0 || !d_x || !d_fval) return fail(ctx, GRC_EINVAL, "orientation fit: NULL buffer");
    if (!(half_width > 0) || max_evals < 1 || max_iter < 1 || !(tol_f >= 0) || !(tol_x >= 0))
        return fail(ctx, GRC_EINVAL, "orientation fit: bad options");
    if (n > (int64_t)INT32_MAX / 4) return fail(ctx, GRC_ECAPACITY, "orientation fit: too many seeds");
    const int64_t T = 4 * n;
    TRY(ensure(ctx, ctx->nm, sizeof(grc::NmSeed) * n));
    TRY(ensure(ctx, ctx->U, sizeof(double) * 9 * T));
    TRY(ensure(ctx, ctx->pos, sizeof(double) * 3 * n));
    TRY(ensure(ctx, ctx->res, sizeof(grc::TrialRes) * T));
    TRY(ensure(ctx, ctx->items, sizeof(longlong4) * T));
    TRY(ensure(ctx, ctx->counter, 8 * sizeof(int)));
    TRY(ensure(ctx, ctx->bad, sizeof(int)));
    if (!ctx->nm_active) CU(cudaMallocHost(&ctx->nm_active, sizeof(int)));
    CU(cudaMemcpyAsync(ctx->pos.p, d_pos, sizeof(double) * 3 * n, cudaMemcpyDeviceToDevice, ctx->stream));
    CU(grc::launch_nm_init((grc::NmSeed *)ctx->nm.p, n, d_x0, half_width, ctx->stream));
    TRY(stage_geo(ctx));
    grc::ScoreBufs b = bufs(ctx);
    grc::Work w{};
    w.items = (const longlong4 *)ctx->items.p;
    w.n_items = T;
    w.n_or = 1;
    w.diag = 1;  // trial t uses orientation t; the voxel comes from items[t]
    int *active = (int *)ctx->bad.p;
    // One graph = kSteps (propose, score, accept) steps plus the running-seed count of the last.
    constexpr int kSteps = 8;
    const int64_t max_steps = 2 * (int64_t)std::min(max_evals, 2 * max_iter) + 8;
    int launches = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    auto enqueue = [&]() -> int {
        for (int k = 0; k < kSteps; ++k) {
            CU(cudaMemsetAsync(active, 0, sizeof(int), ctx->stream));
            CU(grc::launch_nm_propose((grc::NmSeed *)ctx->nm.p, n, max_evals, max_iter, tol_f, tol_x,
                                      (double *)ctx->U.p, (longlong4 *)ctx->items.p, active, ctx->stream));
            cudaError_t e = grc::launch_score(ctx->geo, b, w, ctx->num_sms, ctx->stream, nullptr, nullptr, &launches);
            if (e != cudaSuccess) return fail(ctx, GRC_ECUDA, "orientation fit scorer: %s", cudaGetErrorString(e));
            CU(grc::launch_nm_accept((grc::NmSeed *)ctx->nm.p, n, (const grc::TrialRes *)ctx->res.p, ctx->stream));
        }
        CU(cudaMemcpyAsync(ctx->nm_active, active, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
        return GRC_OK;
    };
    // Device-side loop: one graph whose conditional WHILE node repeats the kSteps body until no seed
    // runs (nm_continue_k sets the condition after each body), so the whole fit is one launch with
    // no host round trip.  Falls back to replaying the body from the host when the runtime cannot
    // build it.
    {
        const int max_bodies = (int)((max_steps + kSteps - 1) / kSteps);
        TRY(ensure(ctx, ctx->nmloop, sizeof(int)));
        int *bodies = (int *)ctx->nmloop.p;  // bodies run, zeroed before the launch
        cudaGraph_t wg = nullptr;
        cudaGraphExec_t wx = nullptr;
        cudaGraphConditionalHandle handle = 0;
        bool built = cudaGraphCreate(&wg, 0) == cudaSuccess &&
                     cudaGraphConditionalHandleCreate(&handle, wg, 1, cudaGraphCondAssignDefault) == cudaSuccess;
        cudaGraphNodeParams cp{};
        cudaGraphNode_t cnode = nullptr;
        if (built) {
            cp.type = cudaGraphNodeTypeConditional;
            cp.conditional.handle = handle;
            cp.conditional.type = cudaGraphCondTypeWhile;
            cp.conditional.size = 1;
            built = cudaGraphAddNode(&cnode, wg, nullptr, 0, &cp) == cudaSuccess;
        }
        if (built) {
            cudaGraph_t body = cp.conditional.phGraph_out[0];
            built = cudaStreamBeginCaptureToGraph(ctx->stream, body, nullptr, nullptr, 0,
                                                  cudaStreamCaptureModeThreadLocal) == cudaSuccess;
            if (built) {
                int brc = GRC_OK;
                for (int k = 0; k < kSteps && brc == GRC_OK; ++k) {
                    if (cudaMemsetAsync(active, 0, sizeof(int), ctx->stream) != cudaSuccess ||
                        grc::launch_nm_propose((grc::NmSeed *)ctx->nm.p, n, max_evals, max_iter, tol_f, tol_x,
                                               (double *)ctx->U.p, (longlong4 *)ctx->items.p, active,
                                               ctx->stream) != cudaSuccess ||
                        grc::launch_score(ctx->geo, b, w, ctx->num_sms, ctx->stream, nullptr, nullptr, &launches) !=
                            cudaSuccess ||
                        grc::launch_nm_accept((grc::NmSeed *)ctx->nm.p, n, (const grc::TrialRes *)ctx->res.p,
                                              ctx->stream) != cudaSuccess)
                        brc = GRC_ECUDA;
                }
                if (brc == GRC_OK &&
                    grc::launch_nm_continue((unsigned long long)handle, active, bodies, max_bodies, ctx->stream) !=
                        cudaSuccess)
                    brc = GRC_ECUDA;
                cudaGraph_t captured = nullptr;
                const bool ended = cudaStreamEndCapture(ctx->stream, &captured) == cudaSuccess;
                built = brc == GRC_OK && ended && cudaGraphInstantiate(&wx, wg, 0) == cudaSuccess;
            }
        }
        if (built) {
            int h_bodies = 0;
            cudaError_t le = cudaMemsetAsync(bodies, 0, sizeof(int), ctx->stream);
            if (le == cudaSuccess) le = cudaGraphLaunch(wx, ctx->stream);
            if (le == cudaSuccess)
                le = cudaMemcpyAsync(&h_bodies, bodies, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream);
            if (le == cudaSuccess) le = cudaStreamSynchronize(ctx->stream);
            cudaGraphExecDestroy(wx);
            cudaGraphDestroy(wg);
            if (le != cudaSuccess) return fail(ctx, GRC_ECUDA, "orientation fit: %s", cudaGetErrorString(le));
            CU(grc::launch_nm_final((const grc::NmSeed *)ctx->nm.p, n, d_x, d_fval, d_evals, d_iters, d_flag,
                                    ctx->stream));
            CU(cudaStreamSynchronize(ctx->stream));
            ctx->stats.trials = (int64_t)h_bodies * kSteps * T;
            ctx->stats.kernel_launches = (int64_t)h_bodies * (kSteps * (2 + launches / kSteps) + 1) + 2;
            ctx->stats.path = 1;
            ctx->stats.device_loop = 1;
            return GRC_OK;
        }
        if (wx) cudaGraphExecDestroy(wx);
        if (wg) cudaGraphDestroy(wg);
        cudaGetLastError();  // the host-driven replay below does the same work
        launches = 0;
    }
    int rc = GRC_OK;
    cudaError_t e = cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        rc = enqueue();
        e = cudaStreamEndCapture(ctx->stream, &graph);
        if (rc == GRC_OK && e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
    }
    if (rc != GRC_OK || e != cudaSuccess) {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        return rc != GRC_OK ? rc : fail(ctx, GRC_ECUDA, "orientation fit graph: %s", cudaGetErrorString(e));
    }
    int64_t steps = 0;
    int graphs = 0;
    for (; steps < max_steps; steps += kSteps) {
        e = cudaGraphLaunch(exec, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        ++graphs;
        if (e != cudaSuccess || *ctx->nm_active == 0) break;
    }
    cudaGraphExecDestroy(exec);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return fail(ctx, GRC_ECUDA, "orientation fit: %s", cudaGetErrorString(e));
    CU(grc::launch_nm_final((const grc::NmSeed *)ctx->nm.p, n, d_x, d_fval, d_evals, d_iters, d_flag, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    ctx->stats.trials = steps * T;
    ctx->stats.kernel_launches = (int64_t)graphs * kSteps * (2 + launches / kSteps) + 2;
    ctx->stats.path = 1;
    return GRC_OK;
}

static_assert(sizeof(grc_spot_pair) == sizeof(grc::PairRec), "grc_spot_pair layout");

int grc_pair_spots(grc_ctx *ctx, const double *d_pos, const double *d_q, int64_t n, const double *d_spots,
                   int64_t n_spots, const int64_t *d_proj_offsets, grc_spot_pair *d_pairs, int64_t max_pairs,
                   int64_t *n_pairs) {
    if (!ctx) return GRC_EINVAL;
    Lock l(ctx);
    if (!n_pairs) return fail(ctx, GRC_EINVAL, "pair: NULL n_pairs");
    *n_pairs = 0;
    TRY(check_ready(ctx));
    ctx->stats = grc_stats{};
    if (n < 0 || n_spots < 0 || max_pairs < 0) return fail(ctx, GRC_EINVAL, "negative size");
    if (n == 0) return GRC_OK;
    if (!d_pos || !d_q || !d_proj_offsets || (n_spots > 0 && !d_spots) || (max_pairs > 0 && !d_pairs))
        return fail(ctx, GRC_EINVAL, "pair: NULL buffer");
    if (n > (int64_t)INT32_MAX || n_spots > (int64_t)INT32_MAX)
        return fail(ctx, GRC_ECAPACITY, "pair: more than 2^31-1 trials or spots");
    const grc::Geo &g = ctx->geo;
    constexpr int kCell = 16;
    const int ncy = (g.detysize + kCell - 1) / kCell, ncz = (g.detzsize + kCell - 1) / kCell;
    const int64_t ncell = (int64_t)g.nrot * ncy * ncz;
    cudaStream_t s = ctx->stream;
    // the projection offsets must describe the spot list
    std::vector<int64_t> off(g.nrot + 1);
    CU(cudaMemcpyAsync(off.data(), d_proj_offsets, sizeof(int64_t) * (g.nrot + 1), cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    if (off[0] != 0 || off[g.nrot] != n_spots)
        return fail(ctx, GRC_EINVAL, "pair: projection offsets must run from 0 to n_spots");
    for (int i = 0; i < g.nrot; ++i)
        if (off[i + 1] < off[i]) return fail(ctx, GRC_EINVAL, "pair: projection offsets decrease at %d", i);
    TRY(ensure(ctx, ctx->U, sizeof(double) * 9 * n));
    TRY(ensure(ctx, ctx->pos, sizeof(double) * 3 * n));
    TRY(ensure(ctx, ctx->cell_cnt, sizeof(int64_t) * (ncell + 1)));
    TRY(ensure(ctx, ctx->cell_off, sizeof(int64_t) * (ncell + 1)));
    TRY(ensure(ctx, ctx->sp_keys, sizeof(int32_t) * (n_spots + 1)));
    TRY(ensure(ctx, ctx->sp_ids, sizeof(int32_t) * (n_spots + 1)));
    TRY(ensure(ctx, ctx->sp_keys2, sizeof(int32_t) * (n_spots + 1)));
    TRY(ensure(ctx, ctx->sp_ids2, sizeof(int32_t) * (n_spots + 1)));
    TRY(ensure(ctx, ctx->pcount, sizeof(unsigned long long)));
    TRY(ensure(ctx, ctx->pr_raw, sizeof(grc::PairRec) * (max_pairs > 0 ? max_pairs : 1)));
    CU(grc::launch_quat_to_u_d(d_q, n, (double *)ctx->U.p, s));
    CU(cudaMemcpyAsync(ctx->pos.p, d_pos, sizeof(double) * 3 * n, cudaMemcpyDeviceToDevice, s));
    CU(cudaMemsetAsync(ctx->cell_cnt.p, 0, sizeof(int64_t) * (ncell + 1), s));
    int end_bit = 1;
    while (end_bit < 31 && ((int64_t)1 << end_bit) < ncell) ++end_bit;
    if (n_spots > 0) {
        CU(grc::launch_spot_keys(d_spots, d_proj_offsets, g.nrot, ncy, ncz, kCell, (int32_t *)ctx->sp_keys.p,
                                 (int32_t *)ctx->sp_ids.p, (int64_t *)ctx->cell_cnt.p, s));
        size_t tb = 0;
        CU(cub::DeviceRadixSort::SortPairs(nullptr, tb, (const int32_t *)ctx->sp_keys.p, (int32_t *)ctx->sp_keys2.p,
                                           (const int32_t *)ctx->sp_ids.p, (int32_t *)ctx->sp_ids2.p, n_spots, 0,
                                           end_bit, s));
        TRY(ensure(ctx, ctx->tmp, tb));
        CU(cub::DeviceRadixSort::SortPairs(ctx->tmp.p, tb, (const int32_t *)ctx->sp_keys.p, (int32_t *)ctx->sp_keys2.p,
                                           (const int32_t *)ctx->sp_ids.p, (int32_t *)ctx->sp_ids2.p, n_spots, 0,
                                           end_bit, s));
    }
    {
        size_t tb = 0;
        CU(cub::DeviceScan::ExclusiveSum(nullptr, tb, (int64_t *)ctx->cell_cnt.p, (int64_t *)ctx->cell_off.p,
                                         ncell + 1, s));
        TRY(ensure(ctx, ctx->tmp, tb));
        CU(cub::DeviceScan::ExclusiveSum(ctx->tmp.p, tb, (int64_t *)ctx->cell_cnt.p, (int64_t *)ctx->cell_off.p,
                                         ncell + 1, s));
    }
    grc::SpotIndex si{d_spots, (const int64_t *)ctx->cell_off.p, (const int32_t *)ctx->sp_ids2.p, ncy, ncz, kCell};
    CU(cudaMemsetAsync(ctx->pcount.p, 0, sizeof(unsigned long long), s));
    TRY(stage_geo(ctx));
    CU(grc::launch_pair(g, bufs(ctx), n, si, (grc::PairRec *)ctx->pr_raw.p, max_pairs,
                        (unsigned long long *)ctx->pcount.p, ctx->num_sms, s));
    unsigned long long cnt = 0;
    CU(cudaMemcpyAsync(&cnt, ctx->pcount.p, sizeof(cnt), cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    *n_pairs = (int64_t)cnt;
    if ((int64_t)cnt > max_pairs) return fail(ctx, GRC_ECAPACITY, "pair: %llu pairs exceed max_pairs", cnt);
    if (cnt > 0) {
        // atomics leave the pairs in arbitrary order: sort by (trial, projection, reflection)
        const int64_t m = (int64_t)cnt;
        TRY(ensure(ctx, ctx->pr_keys, sizeof(int64_t) * m));
        TRY(ensure(ctx, ctx->pr_keys2, sizeof(int64_t) * m));
        TRY(ensure(ctx, ctx->pr_ids, sizeof(int32_t) * m));
        TRY(ensure(ctx, ctx->pr_ids2, sizeof(int32_t) * m));
        CU(grc::launch_pair_keys((const grc::PairRec *)ctx->pr_raw.p, m, g.nrot, g.nhkl, (int64_t *)ctx->pr_keys.p,
                                 (int32_t *)ctx->pr_ids.p, s));
        // keys (trial * nrot + iw) * nhkl + ih are below n * nrot * nhkl: sort only those bits
        const uint64_t key_end = (uint64_t)n * (uint64_t)g.nrot * (uint64_t)g.nhkl;
        int key_bits = 1;
        while (key_bits < 63 && (uint64_t(1) << key_bits) < key_end) ++key_bits;
        size_t tb = 0;
        CU(cub::DeviceRadixSort::SortPairs(nullptr, tb, (const int64_t *)ctx->pr_keys.p, (int64_t *)ctx->pr_keys2.p,
                                           (const int32_t *)ctx->pr_ids.p, (int32_t *)ctx->pr_ids2.p, m, 0, key_bits,
                                           s));
        TRY(ensure(ctx, ctx->tmp, tb));
        CU(cub::DeviceRadixSort::SortPairs(ctx->tmp.p, tb, (const int64_t *)ctx->pr_keys.p, (int64_t *)ctx->pr_keys2.p,
                                           (const int32_t *)ctx->pr_ids.p, (int32_t *)ctx->pr_ids2.p, m, 0, key_bits,
                                           s));
        CU(grc::launch_pair_gather((const grc::PairRec *)ctx->pr_raw.p, (const int32_t *)ctx->pr_ids2.p, m,
                                   (grc::PairRec *)d_pairs, s));
        CU(cudaStreamSynchronize(s));
    }
    ctx->stats.trials = n;
    ctx->stats.kernel_launches = 6 + (cnt > 0 ? 3 : 0);
    return GRC_OK;
}

int grc_last_stats(grc_ctx *ctx, grc_stats *out) {
    if (!ctx || !out) return GRC_EINVAL;
    Lock l(ctx);
    CU(cudaStreamSynchronize(ctx->stream));
    if (ctx->counter.p) {
        int c[8];
        CU(cudaMemcpy(c, ctx->counter.p, sizeof c, cudaMemcpyDeviceToHost));
        ctx->stats.refined = c[4];
        ctx->stats.audit_mismatch = c[5];
        int64_t checked = 0;
        std::memcpy(&checked, c + 6, sizeof checked);
        ctx->stats.audit_checked = checked;
    }
    ctx->stats.score_ms = 0;
    if (ctx->timed_last) {
        float ms = 0;
        if (cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1) == cudaSuccess) ctx->stats.score_ms = ms;
        cudaGetLastError();
    }
    *out = ctx->stats;
    return GRC_OK;
}

int grc_set_path(grc_ctx *ctx, int path) {
    if (!ctx || path < 0 || path > 3) return GRC_EINVAL;
    Lock l(ctx);
    ctx->force_path = path;
    return GRC_OK;
}

int grc_set_timing(grc_ctx *ctx, int enable) {
    if (!ctx) return GRC_EINVAL;
    Lock l(ctx);
    ctx->timing = enable != 0;
    return GRC_OK;
}

int grc_mask_info(grc_ctx *ctx, int64_t *n_distinct, int *code_bits, int64_t *dz, int64_t *dy, int64_t *nrot) {
    if (!ctx) return GRC_EINVAL;
    Lock l(ctx);
    if (!ctx->has_masks) return fail(ctx, GRC_ENOMASK, "no distance map resident");
    if (n_distinct) *n_distinct = ctx->mc.n_distinct;
    if (code_bits) *code_bits = ctx->mc.n_distinct <= 65536 ? 16 : 32;
    if (dz) *dz = ctx->mz;
    if (dy) *dy = ctx->my;
    if (nrot) *nrot = ctx->mrot;
    return GRC_OK;
}

int grc_simulate_spots(grc_ctx *ctx, const float *d_pos, const float *d_U, int64_t n, uint8_t *d_mask) {
    if (!ctx) return GRC_EINVAL;
    Lock l(ctx);
    if (!ctx->has_geo) return fail(ctx, GRC_EINVAL, "no geometry set");
    if (n < 0) return fail(ctx, GRC_EINVAL, "negative size");
    if (n == 0) return GRC_OK;
    if (!d_pos || !d_U || !d_mask) return fail(ctx, GRC_EINVAL, "NULL device buffer");
    TRY(ensure(ctx, ctx->U, sizeof(double) * 9 * n));
    TRY(ensure(ctx, ctx->pos, sizeof(double) * 3 * n));
    TRY(ensure(ctx, ctx->counter, 8 * sizeof(int)));
    CU(grc::launch_f9_to_u(d_U, n, (double *)ctx->U.p, ctx->stream));
    CU(grc::launch_pos_f3(d_pos, n, (double *)ctx->pos.p, ctx->stream));
    TRY(stage_geo(ctx));
    grc::Work w{};
    w.n_or = 1;
    w.chunk = 1;
    w.chunks_per_voxel = 1;
    w.n_items = n;
    w.diag = 1;
    CU(grc::launch_simulate_work(ctx->geo, bufs(ctx), w, ctx->num_sms, d_mask, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    return GRC_OK;
}

int grc_edt(grc_ctx *ctx, const uint8_t *d_mask, int64_t dz, int64_t dy, int64_t nrot, float *d_map) {
    if (!ctx) return GRC_EINVAL;
    Lock l(ctx);
    if (!d_mask || !d_map) return fail(ctx, GRC_EINVAL, "NULL device buffer");
    if (dz < 1 || dy < 1 || nrot < 1) return fail(ctx, GRC_EINVAL, "dimensions must be positive");
    CU(grc::launch_edt(d_mask, dz, dy, nrot, d_map, ctx->stream));
    return GRC_OK;
}

}  // extern "C"

// ---- allocation-free seeding scan ---------------------------------------------------
// Some callers cannot allocate GPU memory at the point where they score: a MEX shim
// living inside MATLAB's gpuArray memory manager, a host framework whose caching
// allocator owns the device, or a tight per-seed loop where cudaMalloc/cudaFree would
// synchronise the whole device.  grc_forward_comp_noalloc serves them from a fixed,
// file-scope device array instead of the context's growable workspace.

namespace {

constexpr int64_t kNoAllocMaxQ = GRC_NOALLOC_MAX_ORIENTATIONS;
constexpr size_t kNaGeo = 0;                                                   // grc::Geo
constexpr size_t kNaCounters = (sizeof(grc::Geo) + 255) & ~size_t(255);       // 8 ints
constexpr size_t kNaPos = kNaCounters + 256;                                   // 3 doubles
constexpr size_t kNaU = kNaPos + 256;                                          // 9 doubles / orientation
constexpr size_t kNaRes = kNaU + sizeof(double) * 9 * kNoAllocMaxQ;            // TrialRes / orientation
constexpr size_t kNaList = kNaRes + sizeof(grc::TrialRes) * kNoAllocMaxQ;      // refine list / orientation
constexpr size_t kNaBytes = kNaList + sizeof(int64_t) * kNoAllocMaxQ;

// Every GPU that loads this library holds this array until the process exits.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNaBytes];

std::mutex g_noalloc_mu;
void *g_noalloc_addr[64];  // device address of g_noalloc_scratch, per device ordinal

// Device address of the scratch array on the current device (looked up once per device).
int noalloc_scratch(grc_ctx *ctx, unsigned char **out) {
    if (ctx->device < 0 || ctx->device >= 64) return fail(ctx, GRC_EINVAL, "noalloc: device ordinal out of range");
    std::lock_guard<std::mutex> g(g_noalloc_mu);
    if (!g_noalloc_addr[ctx->device]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return fail(ctx, GRC_ECUDA, "noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
        g_noalloc_addr[ctx->device] = p;
    }
    *out = (unsigned char *)g_noalloc_addr[ctx->device];
    return GRC_OK;
}

}  // namespace

extern "C" int grc_forward_comp_noalloc(grc_ctx *ctx, const float *pos, const float *d_q, int64_t n_q,
                                        float *d_out) {
    if (!ctx) return GRC_EINVAL;
    Lock l(ctx);
    if (!pos || (n_q > 0 && (!d_q || !d_out))) return fail(ctx, GRC_EINVAL, "noalloc: NULL argument");
    if (n_q < 0) return fail(ctx, GRC_EINVAL, "noalloc: negative orientation count");
    if (n_q > 0) {
        TRY(need_device(ctx, d_q, "noalloc: d_q"));
        TRY(need_device(ctx, d_out, "noalloc: d_out"));
    }
    if (n_q > kNoAllocMaxQ)
        return fail(ctx, GRC_ECAPACITY,
                    "noalloc: %lld orientations exceed the fixed scratch of %lld (GRC_NOALLOC_MAX_ORIENTATIONS); "
                    "split the call or use grc_forward_comp_device",
                    (long long)n_q, (long long)kNoAllocMaxQ);
    TRY(check_ready(ctx));
    if (n_q == 0) return GRC_OK;
    unsigned char *base = nullptr;
    TRY(noalloc_scratch(ctx, &base));
    ctx->stats = grc_stats{};
    // The pinned geometry staging copy is reused; wait until no earlier copy still reads it.
    CU(cudaStreamSynchronize(ctx->stream));
    *ctx->geo_pinned = ctx->geo;
    CU(cudaMemcpyAsync(base + kNaGeo, ctx->geo_pinned, sizeof(grc::Geo), cudaMemcpyHostToDevice, ctx->stream));
    const double p[3] = {pos[0], pos[1], pos[2]};
    CU(cudaMemcpyAsync(base + kNaPos, p, sizeof p, cudaMemcpyHostToDevice, ctx->stream));
    CU(grc::launch_quat_to_u(d_q, n_q, (double *)(base + kNaU), ctx->stream));
    grc::ScoreBufs b{};
    b.geo = (const grc::Geo *)(base + kNaGeo);
    b.rot_cs = (const double2 *)ctx->rot_cs.p;
    b.hkl = (const double *)ctx->hkl.p;
    b.vpos = (const double *)(base + kNaPos);
    b.U = (const double *)(base + kNaU);
    b.codes = ctx->mc.codes;
    b.codes8 = ctx->mc.codes8;
    b.vals = ctx->mc.vals;
    b.res = (grc::TrialRes *)(base + kNaRes);
    b.refine_list = (int64_t *)(base + kNaList);
    b.work_counter = (int *)(base + kNaCounters);  // zeroed by the launchers before their kernels
    grc::Work w{};
    w.n_or = n_q;
    w.chunk = kSeedChunk;
    w.chunks_per_voxel = (n_q + kSeedChunk - 1) / kSeedChunk;
    w.n_items = w.chunks_per_voxel;
    int launches = 0;
    // the kernel the regular entry takes for one voxel: the warp scan from 1/16 of a round (with
    // at least 64 orientations), the per-trial kernel below; both write only the scratch above
    const int64_t round = ctx->force_path == 1 ? 0 : grc::sweep_round_trials(ctx->geo, ctx->num_sms);
    const bool scan = round > 0 && n_q >= 64 && (ctx->force_path >= 2 || n_q >= (round + 15) / 16);
    cudaError_t e = scan ? grc::launch_scan(ctx->geo, b, w, n_q, ctx->num_sms, grc::kScanFull, ctx->stream, nullptr,
                                            nullptr, &launches)
                         : grc::launch_score(ctx->geo, b, w, ctx->num_sms, ctx->stream, nullptr, nullptr, &launches);
    if (e != cudaSuccess) return fail(ctx, GRC_ECUDA, "noalloc scorer launch: %s", cudaGetErrorString(e));
    CU(grc::launch_epi_forward(b.res, n_q, d_out, true, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    ctx->stats.trials = n_q;
    ctx->stats.kernel_launches = launches + 2;
    ctx->stats.path = scan ? 3 : 1;
    return GRC_OK;
}

// ---- batched grower: planned CSR work list, graph capture, autotuned tile -------------
// A grow iteration of grow_unindexed_compete_comp_cuda.m / revise_all_unindexed_voxel_cuda.m
// scores every waiting voxel against its own uneven candidate list.  The plan below builds
// the device work list once, so each iteration is a fixed sequence of kernels with no host
// synchronisation: it can be replayed from a CUDA graph.

struct grc_batch {
    grc_ctx *ctx = nullptr;
    int64_t m = 0, T = 0, n_grain = 0;
    const float *rows5 = nullptr, *euler = nullptr;  // borrowed device arrays
    DevBuf items, torient, tvoxel, res, pos, U, rlist, counter, offsets_h_dummy;
    std::vector<int64_t> offsets;  // host copy of the CSR offsets (m + 1)
    int path = 0, slots = 0;       // chosen tile (0 = by size)
    float *maps[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    int64_t dims[3] = {0, 0, 0};
    DevBuf dims_dev;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int graph_launches = 0;
};

namespace {

uint64_t geo_hash(const grc_ctx *ctx) {
    uint64_t h = 1469598103934665603ull;
    for (float v : ctx->geo_key) {
        uint32_t b;
        std::memcpy(&b, &v, 4);
        h = (h ^ b) * 1099511628211ull;
    }
    return h;
}

std::mutex g_tune_mu;
std::vector<std::pair<uint64_t, std::pair<int, int>>> g_tune_cache;  // geometry hash -> (path, slots)

int batch_enqueue(grc_batch *bt, float *d_out8, float *d_trial_out, int path, int slots, int64_t m_lim,
                  cudaEvent_t e0, cudaEvent_t e1, int *launches) {
    grc_ctx *ctx = bt->ctx;
    const int64_t T = bt->offsets[m_lim];
    grc::ScoreBufs b{};
    b.geo = (const grc::Geo *)ctx->geo_dev.p;
    b.rot_cs = (const double2 *)ctx->rot_cs.p;
    b.hkl = (const double *)ctx->hkl.p;
    b.vpos = (const double *)bt->pos.p;
    b.U = (const double *)bt->U.p;
    b.codes = ctx->mc.codes;
    b.codes8 = ctx->mc.codes8;
    b.vals = ctx->mc.vals;
    b.res = (grc::TrialRes *)bt->res.p;
    b.work_counter = (int *)bt->counter.p;
    b.refine_list = (int64_t *)bt->rlist.p;
    grc::Work w{};
    w.items = (const longlong4 *)bt->items.p;
    w.trial_orient = (const int32_t *)bt->torient.p;
    w.trial_voxel = (const int32_t *)bt->tvoxel.p;
    w.n_items = m_lim;
    cudaError_t e = cudaSuccess;
    if (T > 0) {
        // path 1: per-trial kernel; 2: CTA sweep; 3 (and 0 from half a round on): warp scan
        const int64_t sr = grc::sweep_round_trials(ctx->geo, ctx->num_sms);
        const int use = sr == 0 ? 1 : (path != 0 ? path : (T * 2 >= sr ? 3 : 1));
        if (use == 2)
            e = grc::launch_sweep(ctx->geo, b, w, T, ctx->num_sms, ctx->stream, e0, e1, launches, slots);
        else if (use == 3)
            e = grc::launch_scan(ctx->geo, b, w, T, ctx->num_sms, grc::kScanFull, ctx->stream, e0, e1, launches,
                                 slots);
        else
            e = grc::launch_score(ctx->geo, b, w, ctx->num_sms, ctx->stream, e0, e1, launches);
        if (e != cudaSuccess) return fail(ctx, GRC_ECUDA, "batch scorer launch: %s", cudaGetErrorString(e));
    }
    CU(grc::launch_epi_compete((const grc::TrialRes *)bt->res.p, (const longlong4 *)bt->items.p,
                               (const int32_t *)bt->torient.p, m_lim, bt->euler, d_out8, d_trial_out, ctx->stream));
    ++*launches;
    if (bt->maps[0] || bt->maps[1] || bt->maps[2] || bt->maps[3] || bt->maps[4]) {
        CU(grc::launch_apply_compete(d_out8, bt->rows5, m_lim, bt->dims, bt->maps[0], bt->maps[1], bt->maps[2],
                                     bt->maps[3], bt->maps[4], ctx->stream));
        ++*launches;
    }
    return GRC_OK;
}

}  // namespace

extern "C" int grc_batch_create(grc_ctx *ctx, const float *d_rows5, int64_t m, const float *d_id, int64_t n_neigb,
                                const float *d_euler, int64_t n_grain, const float *param1, grc_batch **out) {
    if (!ctx || !out) return GRC_EINVAL;
    *out = nullptr;
    Lock l(ctx);
    TRY(check_ready(ctx));
    if (!param1 || m < 1 || !d_rows5 || !d_euler || n_grain < 1 || n_grain > (int64_t)INT32_MAX || n_neigb < 0)
        return fail(ctx, GRC_EINVAL, "batch: bad arguments");
    double p1[14] = {0};
    for (int i = 0; i < 11; ++i) {
        if (!std::isfinite(param1[i])) return fail(ctx, GRC_EINVAL, "param1(%d) is not finite", i + 1);
        p1[i] = param1[i];
    }
    grc_batch *bt = new grc_batch();
    bt->ctx = ctx;
    bt->m = m;
    bt->n_grain = n_grain;
    bt->rows5 = d_rows5;
    bt->euler = d_euler;
    auto bail = [&](int rc) {
        DevBuf *all[] = {&bt->items, &bt->torient, &bt->tvoxel, &bt->res, &bt->pos, &bt->U, &bt->rlist,
                         &bt->counter, &bt->dims_dev};
        for (DevBuf *d : all) cudaFree(d->p);
        delete bt;
        return rc;
    };
    int rc;
    if ((rc = ensure(ctx, ctx->p1, sizeof(p1))) || (rc = ensure(ctx, bt->U, sizeof(double) * 9 * n_grain)) ||
        (rc = ensure(ctx, bt->pos, sizeof(double) * 3 * m)) || (rc = ensure(ctx, ctx->counts, sizeof(int64_t) * m)) ||
        (rc = ensure(ctx, ctx->offsets, sizeof(int64_t) * m)) || (rc = ensure(ctx, bt->items, sizeof(longlong4) * m)) ||
        (rc = ensure(ctx, ctx->bad, sizeof(int))) || (rc = ensure(ctx, bt->counter, 8 * sizeof(int))))
        return bail(rc);
    cudaStream_t s = ctx->stream;
    size_t tmp_bytes = 0;
    int64_t last_off = 0, last_cnt = 0;
    int hbad = 0;
    cudaError_t e;
#define BCK(x)                                                                                  \
    do {                                                                                        \
        e = (x);                                                                                \
        if (e != cudaSuccess) return bail(fail(ctx, GRC_ECUDA, "batch: %s", cudaGetErrorString(e))); \
    } while (0)
    BCK(cudaMemcpyAsync(ctx->p1.p, p1, sizeof(p1), cudaMemcpyHostToDevice, s));
    BCK(cudaMemsetAsync(ctx->bad.p, 0, sizeof(int), s));
    BCK(grc::launch_euler_to_u(d_euler, n_grain, (double *)bt->U.p, s));
    BCK(grc::launch_pos_rows(d_rows5, 5, m, (const double *)ctx->p1.p, (double *)bt->pos.p, s));
    BCK(grc::launch_csr_counts(d_rows5, m, (int64_t *)ctx->counts.p, s));
    BCK(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, (int64_t *)ctx->counts.p, (int64_t *)ctx->offsets.p, m, s));
    if ((rc = ensure(ctx, ctx->tmp, tmp_bytes))) return bail(rc);
    BCK(cub::DeviceScan::ExclusiveSum(ctx->tmp.p, tmp_bytes, (int64_t *)ctx->counts.p, (int64_t *)ctx->offsets.p, m, s));
    bt->offsets.resize(m + 1);
    BCK(cudaMemcpyAsync(bt->offsets.data(), ctx->offsets.p, sizeof(int64_t) * m, cudaMemcpyDeviceToHost, s));
    BCK(cudaMemcpyAsync(&last_cnt, (int64_t *)ctx->counts.p + (m - 1), 8, cudaMemcpyDeviceToHost, s));
    BCK(cudaStreamSynchronize(s));
    last_off = bt->offsets[m - 1];
    bt->T = last_off + last_cnt;
    bt->offsets[m] = bt->T;
    const int64_t T = bt->T > 0 ? bt->T : 1;
    if ((rc = ensure(ctx, bt->torient, sizeof(int32_t) * T)) || (rc = ensure(ctx, bt->tvoxel, sizeof(int32_t) * T)) ||
        (rc = ensure(ctx, bt->res, sizeof(grc::TrialRes) * T)) || (rc = ensure(ctx, bt->rlist, sizeof(int64_t) * T)))
        return bail(rc);
    BCK(grc::launch_csr_fill(d_rows5, m, (const int64_t *)ctx->offsets.p, d_id, n_neigb, n_grain,
                             (longlong4 *)bt->items.p, (int32_t *)bt->torient.p, (int32_t *)bt->tvoxel.p,
                             (int *)ctx->bad.p, s));
    BCK(cudaMemcpyAsync(&hbad, ctx->bad.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    BCK(cudaStreamSynchronize(s));
#undef BCK
    if (hbad & 1) return bail(fail(ctx, GRC_EINVAL, "batch: a [first,last] range lies outside id_neigb_all"));
    if (hbad & 2) return bail(fail(ctx, GRC_EINVAL, "batch: a grain id lies outside the Euler table"));
    if ((rc = stage_geo(ctx))) return bail(rc);
    if (cudaStreamSynchronize(s) != cudaSuccess) return bail(fail(ctx, GRC_ECUDA, "batch: sync failed"));
    {
        std::lock_guard<std::mutex> g(g_tune_mu);
        const uint64_t h = geo_hash(ctx);
        for (auto &kv : g_tune_cache)
            if (kv.first == h) {
                bt->path = kv.second.first;
                bt->slots = kv.second.second;
            }
    }
    *out = bt;
    return GRC_OK;
}

extern "C" int grc_batch_set_maps(grc_batch *bt, const int64_t *dims, float *d_completeness, float *d_grain_id,
                                  float *d_dismedian, float *d_ninter, float *d_visitflag) {
    if (!bt || !dims) return GRC_EINVAL;
    Lock l(bt->ctx);
    for (int i = 0; i < 3; ++i) {
        if (dims[i] < 1) return fail(bt->ctx, GRC_EINVAL, "batch maps: dimensions must be positive");
        bt->dims[i] = dims[i];
    }
    bt->maps[0] = d_completeness;
    bt->maps[1] = d_grain_id;
    bt->maps[2] = d_dismedian;
    bt->maps[3] = d_ninter;
    bt->maps[4] = d_visitflag;
    return GRC_OK;
}

extern "C" int grc_batch_run(grc_batch *bt, float *d_out8, float *d_trial_out) {
    if (!bt || !d_out8) return GRC_EINVAL;
    grc_ctx *ctx = bt->ctx;
    Lock l(ctx);
    ctx->stats = grc_stats{};
    int launches = 0;
    cudaEvent_t e0 = ctx->timing ? ctx->ev0 : nullptr, e1 = ctx->timing ? ctx->ev1 : nullptr;
    TRY(batch_enqueue(bt, d_out8, d_trial_out, bt->path, bt->slots, bt->m, e0, e1, &launches));
    ctx->timed_last = ctx->timing;
    ctx->stats.trials = bt->T;
    ctx->stats.kernel_launches = launches;
    return GRC_OK;
}

extern "C" int grc_batch_capture(grc_batch *bt, float *d_out8) {
    if (!bt || !d_out8) return GRC_EINVAL;
    grc_ctx *ctx = bt->ctx;
    Lock l(ctx);
    CU(cudaStreamSynchronize(ctx->stream));
    if (bt->exec) {
        cudaGraphExecDestroy(bt->exec);
        bt->exec = nullptr;
    }
    if (bt->graph) {
        cudaGraphDestroy(bt->graph);
        bt->graph = nullptr;
    }
    CU(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    int launches = 0;
    const int rc = batch_enqueue(bt, d_out8, nullptr, bt->path, bt->slots, bt->m, nullptr, nullptr, &launches);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
    if (rc != GRC_OK) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess) return fail(ctx, GRC_ECUDA, "batch capture: %s", cudaGetErrorString(e));
    bt->graph = g;
    CU(cudaGraphInstantiate(&bt->exec, g, 0));
    bt->graph_launches = launches;
    return GRC_OK;
}

extern "C" int grc_batch_replay(grc_batch *bt) {
    if (!bt) return GRC_EINVAL;
    grc_ctx *ctx = bt->ctx;
    Lock l(ctx);
    if (!bt->exec) return fail(ctx, GRC_EINVAL, "batch: no captured graph");
    ctx->stats = grc_stats{};
    CU(cudaGraphLaunch(bt->exec, ctx->stream));
    ctx->stats.trials = bt->T;
    ctx->stats.kernel_launches = bt->graph_launches;
    return GRC_OK;
}

extern "C" int grc_batch_autotune(grc_batch *bt, float *d_out8, int64_t max_voxels, int *path_out, int *slots_out,
                                  double *ms_out) {
    if (!bt || !d_out8) return GRC_EINVAL;
    grc_ctx *ctx = bt->ctx;
    Lock l(ctx);
    int64_t m_lim = bt->m;
    if (max_voxels > 0 && max_voxels < m_lim) m_lim = max_voxels;
    struct Cand {
        int path, slots;
    };
    const Cand cands[] = {{1, 0}, {2, 16}, {2, 32}, {2, 48}, {2, 64}, {3, 16}, {3, 32}, {3, 48}, {3, 64}};
    cudaEvent_t a, z;
    CU(cudaEventCreate(&a));
    CU(cudaEventCreate(&z));
    double best = 1e300;
    Cand pick{0, 0};
    int rc = GRC_OK;
    for (const Cand &c : cands) {
        if (c.path >= 2 && grc::sweep_round_trials(ctx->geo, ctx->num_sms) == 0) continue;
        double t_best = 1e300;
        for (int rep = 0; rep < 2 && rc == GRC_OK; ++rep) {
            int launches = 0;
            cudaEventRecord(a, ctx->stream);
            rc = batch_enqueue(bt, d_out8, nullptr, c.path, c.slots, m_lim, nullptr, nullptr, &launches);
            cudaEventRecord(z, ctx->stream);
            if (cudaEventSynchronize(z) != cudaSuccess) rc = fail(ctx, GRC_ECUDA, "autotune: sync failed");
            float ms = 0;
            cudaEventElapsedTime(&ms, a, z);
            if (rep > 0 || true) t_best = std::min(t_best, (double)ms);
        }
        if (rc != GRC_OK) break;
        if (t_best < best) {
            best = t_best;
            pick = c;
        }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(z);
    if (rc != GRC_OK) return rc;
    bt->path = pick.path;
    bt->slots = pick.slots;
    {
        std::lock_guard<std::mutex> g(g_tune_mu);
        const uint64_t h = geo_hash(ctx);
        bool found = false;
        for (auto &kv : g_tune_cache)
            if (kv.first == h) {
                kv.second = {pick.path, pick.slots};
                found = true;
            }
        if (!found) g_tune_cache.push_back({h, {pick.path, pick.slots}});
    }
    if (path_out) *path_out = pick.path;
    if (slots_out) *slots_out = pick.slots;
    if (ms_out) *ms_out = best;
    return GRC_OK;
}

extern "C" int grc_batch_info(grc_batch *bt, int64_t *n_voxels, int64_t *n_trials, int *path, int *slots) {
    if (!bt) return GRC_EINVAL;
    if (n_voxels) *n_voxels = bt->m;
    if (n_trials) *n_trials = bt->T;
    if (path) *path = bt->path;
    if (slots) *slots = bt->slots;
    return GRC_OK;
}

extern "C" int grc_batch_destroy(grc_batch *bt) {
    if (!bt) return GRC_EINVAL;
    {
        Lock l(bt->ctx);
        cudaStreamSynchronize(bt->ctx->stream);
        if (bt->exec) cudaGraphExecDestroy(bt->exec);
        if (bt->graph) cudaGraphDestroy(bt->graph);
        DevBuf *all[] = {&bt->items, &bt->torient, &bt->tvoxel, &bt->res, &bt->pos, &bt->U, &bt->rlist,
                         &bt->counter, &bt->dims_dev};
        for (DevBuf *d : all) cudaFree(d->p);
    }
    delete bt;
    return GRC_OK;
}


// ---- spot-centroid residual, its derivatives and the fits ---------------------------
namespace {

int fit_prepare(grc_ctx *ctx, const double *geo10, grc::FitFixed *fx) {
    if (!ctx->has_geo) return fail(ctx, GRC_EINVAL, "fit: no geometry set");
    const grc::Geo &g = ctx->geo;
    for (int i = 0; i < 9; ++i) {
        fx->S[i] = g.S[i];
        fx->B[i] = g.B[i];
    }
    fx->pxy = g.pxy;
    fx->pxz = g.pxz;
    fx->dety0 = g.dety0;
    fx->detz0 = g.detz0;
    fx->lmin = g.lmin;
    fx->lmax = g.lmax;
    fx->cbmax = g.cbmax;
    fx->detysize = g.detysize;
    fx->detzsize = g.detzsize;
    fx->nrot = g.nrot;
    fx->nhkl = g.nhkl;
    fx->rot_cs = (const double2 *)ctx->rot_cs.p;
    fx->hkl = (const double *)ctx->hkl.p;
    if (geo10) {
        for (int i = 0; i < 10; ++i)
            if (!std::isfinite(geo10[i])) return fail(ctx, GRC_EINVAL, "fit: geometry parameter %d is not finite", i);
        TRY(ensure(ctx, ctx->fgeo, sizeof(double) * 10));
        CU(cudaMemcpyAsync(ctx->fgeo.p, geo10, sizeof(double) * 10, cudaMemcpyHostToDevice, ctx->stream));
    }
    return GRC_OK;
}

grc::SpotList spots_of(const int32_t *g, const int32_t *w, const int32_t *h, const double *uv, int64_t n) {
    grc::SpotList sp;
    sp.grain = const_cast<int32_t *>(g);
    sp.iw = const_cast<int32_t *>(w);
    sp.ih = const_cast<int32_t *>(h);
    sp.uv = const_cast<double *>(uv);
    sp.n = n;
    return sp;
}

}  // namespace

extern "C" int grc_fit_spot_count(grc_ctx *ctx, const double *geo10, const double *d_grains, int64_t n_grains,
                                  int64_t *d_counts) {
    if (!ctx) return GRC_EINVAL;
    Lock l(ctx);
    if (!geo10 || !d_grains || !d_counts || n_grains < 0) return fail(ctx, GRC_EINVAL, "fit: bad arguments");
    grc::FitFixed fx;
    TRY(fit_prepare(ctx, geo10, &fx));
    if (n_grains == 0) return GRC_OK;
    CU(grc::fit_spots_count(fx, d_grains, (const double *)ctx->fgeo.p, n_grains, d_counts, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    return GRC_OK;
}

extern "C" int grc_fit_spot_fill(grc_ctx *ctx, const double *geo10, const double *d_grains, int64_t n_grains,
                                 const int64_t *d_offsets, int32_t *d_grain, int32_t *d_iw, int32_t *d_ih,
                                 double *d_uv) {
    if (!ctx) return GRC_EINVAL;
    Lock l(ctx);
    if (!geo10 || !d_grains || !d_offsets || !d_grain || !d_iw || !d_ih || !d_uv || n_grains < 0)
        return fail(ctx, GRC_EINVAL, "fit: bad arguments");
    grc::FitFixed fx;
    TRY(fit_prepare(ctx, geo10, &fx));
    if (n_grains == 0) return GRC_OK;
    CU(grc::fit_spots_fill(fx, d_grains, (const double *)ctx->fgeo.p, n_grains, d_offsets,
                           spots_of(d_grain, d_iw, d_ih, d_uv, 0), ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    return GRC_OK;
}

extern "C" int grc_centroid_residual_adjoint(grc_ctx *ctx, int mode, const double *geo10, const double *d_grains,
                                             const int32_t *d_grain, const int32_t *d_iw, const int32_t *d_ih,
                                             const double *d_uv, int64_t n_spots, double *d_res, double *d_jac) {
    if (!ctx) return GRC_EINVAL;
    Lock l(ctx);
    if (mode != 0 && mode != 1) return fail(ctx, GRC_EINVAL, "fit: mode must be 0 (grain) or 1 (geometry)");
    if (!geo10 || !d_grains || n_spots < 0 || (n_spots > 0 && (!d_grain || !d_iw || !d_ih || !d_uv || !d_res || !d_jac)))
        return fail(ctx, GRC_EINVAL, "fit: bad arguments");
    grc::FitFixed fx;
    TRY(fit_prepare(ctx, geo10, &fx));
    if (n_spots == 0) return GRC_OK;
    CU(grc::fit_residual_jacobian(fx, mode, d_grains, (const double *)ctx->fgeo.p,
                                  spots_of(d_grain, d_iw, d_ih, d_uv, n_spots), d_res, d_jac, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    return GRC_OK;
}

extern "C" int grc_fit_grains_lm(grc_ctx *ctx, const double *geo10, double *d_grains, int64_t n_grains,
                                 const int32_t *d_grain, const int32_t *d_iw, const int32_t *d_ih, const double *d_uv,
                                 int64_t n_spots, const int64_t *d_offsets, double *d_lambda, int iters,
                                 int *n_improved) {
    if (!ctx) return GRC_EINVAL;
    Lock l(ctx);
    if (!geo10 || !d_grains || !d_offsets || !d_lambda || n_grains < 1 || iters < 0)
        return fail(ctx, GRC_EINVAL, "fit: bad arguments");
    grc::FitFixed fx;
    TRY(fit_prepare(ctx, geo10, &fx));
    TRY(ensure(ctx, ctx->fne, sizeof(double) * 29 * n_grains));
    TRY(ensure(ctx, ctx->ftrial, sizeof(double) * 6 * n_grains));
    TRY(ensure(ctx, ctx->fcost0, sizeof(double) * 2 * n_grains));
    TRY(ensure(ctx, ctx->fcost1, sizeof(double) * 2 * n_grains));
    TRY(ensure(ctx, ctx->fimp, sizeof(int)));
    const grc::SpotList sp = spots_of(d_grain, d_iw, d_ih, d_uv, n_spots);
    const double *g10 = (const double *)ctx->fgeo.p;
    int improved = 0;
    for (int it = 0; it < iters; ++it) {
        CU(cudaMemsetAsync(ctx->fimp.p, 0, sizeof(int), ctx->stream));
        CU(grc::fit_grain_normal(fx, d_grains, g10, sp, d_offsets, n_grains, (double *)ctx->fne.p, ctx->stream));
        CU(grc::fit_grain_cost(fx, d_grains, g10, sp, d_offsets, n_grains, (double *)ctx->fcost0.p, ctx->stream));
        CU(grc::fit_grain_lm_propose(d_grains, (const double *)ctx->fne.p, d_lambda, n_grains,
                                     (double *)ctx->ftrial.p, ctx->stream));
        CU(grc::fit_grain_cost(fx, (const double *)ctx->ftrial.p, g10, sp, d_offsets, n_grains,
                               (double *)ctx->fcost1.p, ctx->stream));
        CU(grc::fit_grain_lm_accept(d_grains, (const double *)ctx->ftrial.p, (const double *)ctx->fcost0.p,
                                    (const double *)ctx->fcost1.p, d_lambda, n_grains, (int *)ctx->fimp.p,
                                    ctx->stream));
        CU(cudaMemcpyAsync(&improved, ctx->fimp.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
        CU(cudaStreamSynchronize(ctx->stream));
        if (improved == 0) break;
    }
    if (n_improved) *n_improved = improved;
    return GRC_OK;
}

extern "C" int grc_fit_grains_nm(grc_ctx *ctx, const double *geo10, double *d_grains, int64_t n_grains,
                                 const int32_t *d_grain, const int32_t *d_iw, const int32_t *d_ih, const double *d_uv,
                                 int64_t n_spots, const int64_t *d_offsets, const double *half_width, int max_evals,
                                 int checkpoint, double *d_trace, int n_ck) {
    if (!ctx) return GRC_EINVAL;
    Lock l(ctx);
    if (!geo10 || !d_grains || !d_offsets || !half_width || n_grains < 1 || max_evals < 7 ||
        (d_trace && (checkpoint < 1 || n_ck < 1)))
        return fail(ctx, GRC_EINVAL, "fit: bad arguments");
    grc::FitFixed fx;
    TRY(fit_prepare(ctx, geo10, &fx));
    TRY(ensure(ctx, ctx->fhw, sizeof(double) * 6));
    CU(cudaMemcpyAsync(ctx->fhw.p, half_width, sizeof(double) * 6, cudaMemcpyHostToDevice, ctx->stream));
    CU(grc::fit_grain_nm(fx, d_grains, (const double *)ctx->fgeo.p, spots_of(d_grain, d_iw, d_ih, d_uv, n_spots),
                         d_offsets, n_grains, (const double *)ctx->fhw.p, max_evals, checkpoint, d_trace,
                         d_trace ? n_ck : 0, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    return GRC_OK;
}

extern "C" int grc_fit_grains_rms(grc_ctx *ctx, const double *geo10, const double *d_grains, const double *d_truth,
                                  int64_t n_grains, const int32_t *d_grain, const int32_t *d_iw, const int32_t *d_ih,
                                  const double *d_uv, int64_t n_spots, const int64_t *d_offsets, double *d_rms) {
    if (!ctx) return GRC_EINVAL;
    Lock l(ctx);
    if (!geo10 || !d_grains || !d_truth || !d_offsets || !d_rms || n_grains < 1)
        return fail(ctx, GRC_EINVAL, "fit: bad arguments");
    grc::FitFixed fx;
    TRY(fit_prepare(ctx, geo10, &fx));
    CU(grc::fit_grain_rms(fx, d_grains, d_truth, (const double *)ctx->fgeo.p,
                          spots_of(d_grain, d_iw, d_ih, d_uv, n_spots), d_offsets, n_grains, d_rms, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    return GRC_OK;
}

extern "C" int grc_fit_geometry_lm(grc_ctx *ctx, double *d_starts, int n_starts, const double *d_grains,
                                   const int32_t *d_grain, const int32_t *d_iw, const int32_t *d_ih, const double *d_uv,
                                   int64_t n_spots, double *d_lambda, int iters, int *n_improved) {
    if (!ctx) return GRC_EINVAL;
    Lock l(ctx);
    if (!d_starts || !d_grains || !d_lambda || n_starts < 1 || n_starts > 65535 || iters < 0 || n_spots < 1)
        return fail(ctx, GRC_EINVAL, "fit: bad arguments");
    grc::FitFixed fx;
    TRY(fit_prepare(ctx, nullptr, &fx));
    TRY(ensure(ctx, ctx->fne, sizeof(double) * 67 * n_starts));
    TRY(ensure(ctx, ctx->ftrial, sizeof(double) * 10 * n_starts));
    TRY(ensure(ctx, ctx->fcost0, sizeof(double) * 2 * n_starts));
    TRY(ensure(ctx, ctx->fcost1, sizeof(double) * 2 * n_starts));
    TRY(ensure(ctx, ctx->fimp, sizeof(int)));
    const grc::SpotList sp = spots_of(d_grain, d_iw, d_ih, d_uv, n_spots);
    int improved = 0;
    for (int it = 0; it < iters; ++it) {
        CU(cudaMemsetAsync(ctx->fimp.p, 0, sizeof(int), ctx->stream));
        CU(grc::fit_geo_normal(fx, d_grains, d_starts, n_starts, sp, (double *)ctx->fne.p, ctx->num_sms, ctx->stream));
        CU(grc::fit_geo_cost(fx, d_grains, d_starts, n_starts, sp, (double *)ctx->fcost0.p, ctx->num_sms, ctx->stream));
        CU(grc::fit_geo_lm_propose(d_starts, (const double *)ctx->fne.p, d_lambda, n_starts, (double *)ctx->ftrial.p,
                                   ctx->stream));
        CU(grc::fit_geo_cost(fx, d_grains, (const double *)ctx->ftrial.p, n_starts, sp, (double *)ctx->fcost1.p,
                             ctx->num_sms, ctx->stream));
        CU(grc::fit_geo_lm_accept(d_starts, (const double *)ctx->ftrial.p, (const double *)ctx->fcost0.p,
                                  (const double *)ctx->fcost1.p, d_lambda, n_starts, (int *)ctx->fimp.p, ctx->stream));
        CU(cudaMemcpyAsync(&improved, ctx->fimp.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
        CU(cudaStreamSynchronize(ctx->stream));
        if (improved == 0) break;
    }
    if (n_improved) *n_improved = improved;
    return GRC_OK;
}

extern "C" int grc_fit_geometry_cost(grc_ctx *ctx, const double *d_points, int n_points, const double *d_grains,
                                     const int32_t *d_grain, const int32_t *d_iw, const int32_t *d_ih,
                                     const double *d_uv, int64_t n_spots, double *d_cost) {
    if (!ctx) return GRC_EINVAL;
    Lock l(ctx);
    if (!d_points || !d_grains || !d_cost || n_points < 1 || n_points > 65535 || n_spots < 1)
        return fail(ctx, GRC_EINVAL, "fit: bad arguments");
    grc::FitFixed fx;
    TRY(fit_prepare(ctx, nullptr, &fx));
    CU(grc::fit_geo_cost(fx, d_grains, d_points, n_points, spots_of(d_grain, d_iw, d_ih, d_uv, n_spots), d_cost,
                         ctx->num_sms, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    return GRC_OK;
}

extern "C" int grc_fit_geometry_rms(grc_ctx *ctx, const double *d_starts, int n_starts, const double *geo_truth10,
                                    const double *d_grains, const int32_t *d_grain, const int32_t *d_iw,
                                    const int32_t *d_ih, const double *d_uv, int64_t n_spots, double *d_acc) {
    if (!ctx) return GRC_EINVAL;
    Lock l(ctx);
    if (!d_starts || !geo_truth10 || !d_grains || !d_acc || n_starts < 1 || n_starts > 65535 || n_spots < 1)
        return fail(ctx, GRC_EINVAL, "fit: bad arguments");
    grc::FitFixed fx;
    TRY(fit_prepare(ctx, geo_truth10, &fx));
    CU(grc::fit_geo_rms(fx, d_grains, d_starts, n_starts, (const double *)ctx->fgeo.p,
                        spots_of(d_grain, d_iw, d_ih, d_uv, n_spots), d_acc, ctx->num_sms, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    return GRC_OK;
}
