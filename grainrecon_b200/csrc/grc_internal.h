// grc_internal.h -- types shared by the scorer kernels and the C-ABI layer.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace grc {

// Histogram width of the first scoring pass: distance-map codes below kHistBins
// are counted exactly in shared memory; a trial whose median rank falls on a
// larger code is finished by the radix refine kernel.
constexpr int kHistBins = 1024;
constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kQueueCap = 32 + 32 * 4;  // one 32-item batch in flight + 4 reflection slots per lane
constexpr int kFallbackCap = 64;       // ambiguous items awaiting the FP64 path (< 32 + 32)

// Scalar geometry of one scorer call, FP64 (promoted from the float32 MEX
// arguments).  Field names follow forward_comp.m.
struct Geo {
    double lss, lsd, p0y, p0z, dety00, detz00, pxy, pxz, rao;
    double dety0, detz0;
    double lmin, lmax;       // wavelength window [A]
    double cbmax;            // cos((90+4*thetamax) deg), or -2 when that angle is >= 180 deg
    double bsy0, bsy1, bsz0, bsz1;
    double S[9], B[9], R[9]; // row-major
    // FP32 copies for the fast landing chain
    float Rf[9];
    float Ruf[2], Rvf[2];    // R[4]/pxy, R[7]/pxy and R[5]/pxz, R[8]/pxz (ray K -> pixel u, v)
    float dety0f, detz0f, rpxyf, rpxzf;
    float bsy0f, bsy1f, bsz0f, bsz1f;
    float lo4pif, hi4pif, cbmaxf;   // lambda_min/(4 pi), lambda_max/(4 pi), cos(beta_max)
    int nhkl, nrot, detysize, detzsize;
    uint32_t n_hit;          // codes [0, n_hit) are "dis <= threshold"
    uint32_t n_vals;         // entries of the code -> value table
    int code_bits;           // bits of the largest code (radix passes of the refine kernel)
    int64_t plane;           // detysize * detzsize
};

// Per-trial result of the scoring pass.  median is NaN while the exact radix
// refine pass still has to produce it.
struct TrialRes {
    int32_t simu;
    int32_t inter;
    double median;
};

// Work enumeration.  Explicit: items[i] = {voxel, t_begin, t_end} and
// trial_orient[t] = orientation index.  Implicit (items == nullptr):
// n_vox voxels x n_or orientations in chunks of `chunk`, trial t = v*n_or + o.
// diag != 0: trial t uses orientation t (one orientation per voxel).
struct Work {
    const longlong4 *items;
    const int32_t *trial_orient;
    const int32_t *trial_voxel;   // explicit voxel per trial (sweep kernel), or nullptr
    int64_t n_items;
    int64_t n_or;
    int64_t chunks_per_voxel;
    int32_t chunk;
    int32_t diag;
    // Explicit lists: the most voxel-run starts (t = 0 or trial_voxel[t] != trial_voxel[t-1]) in
    // any aligned block of 32 trials, or 0 when unknown.  Bounds the distinct voxels a sweep tile
    // meets, so seed-major lists need one omega-row set per voxel, not one per trial.
    int32_t starts_per_32;
};

struct ScoreBufs {
    const Geo *geo;           // device copy of the kernel's Geo (read by the exact FP64 path)
    const double2 *rot_cs;    // cos/sin of every omega
    const double *hkl;        // 3*nhkl
    const double *vpos;       // 3 per voxel [mm]
    const double *U;          // 9 per orientation
    const void *codes;        // rank codes of the distance map
    const uint8_t *codes8;    // the same codes saturated at 255 (sweep kernel)
    const float *vals;        // code -> distance value
    int64_t *refine_list;     // trials whose median needs the exact refine pass (sweep kernel)
    TrialRes *res;
    int *work_counter;        // 8 ints: [0..1] main-pass item counter (u64), [2..3] refine-pass
                              // item counter (u64), [4] trials left for the refine pass
    const uint32_t *bits;     // hit mask, 1 bit per pixel (code < n_hit): plane_words words per
                              // projection, pixel (dety-1)*detzsize + (detz-1) at bit p&31 of word p>>5
    int64_t plane_words;
    unsigned long long *group_key;  // optional first-maximum key per group of group_size trials
    int64_t group_size;
};

size_t score_smem_bytes(int nrot, int nhkl);
size_t refine_smem_bytes(int nrot, int nhkl);
// Enqueue the scoring pass (+ refine pass) on `s`.  Returns a cudaError_t.
cudaError_t launch_score(const Geo &g, const ScoreBufs &b, const Work &w, int num_sms, cudaStream_t s,
                         cudaEvent_t ev0, cudaEvent_t ev1, int *launches);
// Trials one round of the projection-window sweep holds (grid x slots); 0 if the sweep
// cannot serve this geometry.
int64_t sweep_round_trials(const Geo &g, int num_sms);
// Enqueue the radix refine pass over the trials a sweep listed (work_counter[4] of them).
cudaError_t launch_refine_list(const Geo &g, const ScoreBufs &b, const Work &w, int num_sms, cudaStream_t s);
// Trial scan with one trial per warp at a time (grc_scan.cu).  mode 0: counts and the exact median
// from the 8-bit codes (+ the list refine pass); mode 1: counts only, from the bit-packed hit mask
// (median NaN).  With b.group_key set, the first maximum of completeness of every group of
// b.group_size consecutive trials is folded into group_key (group_key_of).
constexpr int kScanFull = 0, kScanComp = 1;
int64_t scan_round_trials(const Geo &g, int num_sms);

// Launch-configuration helpers shared by the window kernels' launchers.  occupancy_for: resident
// CTAs per SM of `fn` with 256 threads and `smem` bytes of dynamic shared memory, cached per
// (device, kernel, size); allow_smem: raises the kernel's dynamic shared-memory limit to at least
// `smem` (each only calls the runtime the first time it meets a kernel and size).
cudaError_t occupancy_for(const void *fn, size_t smem, int *per_sm);
cudaError_t allow_smem(const void *fn, size_t smem);
cudaError_t launch_scan(const Geo &g, const ScoreBufs &b, const Work &w, int64_t n_trials, int num_sms, int mode,
                        cudaStream_t s, cudaEvent_t ev0, cudaEvent_t ev1, int *launches, int max_slots = 0);
// Seeding-stage ordering (grc_select.cu).  top_rows: per group of gsize rows, the indices of the
// first n_top rows of sortrows(.., 'descend') on completeness (NaN first, stable) -- from a float
// column (vals, stride floats apart) or, with vals NULL, from the trial results.  n_top <= 4096.
cudaError_t launch_top_rows(const float *vals, const TrialRes *res, int64_t stride, int64_t n_groups, int64_t gsize,
                            int n_top, int32_t *idx, cudaStream_t s);
// out[(g*n_top + k)*row_len + c] = source row idx[g*n_top + k] + g*src_group_stride (float rows
// widened to double, or double rows).
cudaError_t launch_gather_rows(const int32_t *idx, int64_t n_groups, int n_top, int64_t gsize, const float *src_f,
                               const double *src_d, int64_t src_group_stride, int row_len, double *out,
                               cudaStream_t s);
// out[g*n_top + r] = src[g*src_stride + idx[g*n_top + r]].
cudaError_t launch_gather_floats(const int32_t *idx, int64_t n_groups, int n_top, int64_t gsize, const float *src,
                                 int64_t src_stride, float *out, cudaStream_t s);
// x0[(s*n_x0 + j)*3 + c] = rows[(s*k + j)*4 + 1 + c]: (b, c, d) of each seed's first n_x0 rows.
cudaError_t launch_take_x0(const double *rows, int64_t n, int k, int n_x0, double *x0, cudaStream_t s);
// ori_local_sampling grids of n_cand quaternions (4 doubles each): local_grid_rows(nr) rows per
// candidate in unique(q,'rows') order into out, and (optional) the same rows rounded to float32,
// widened back to double (out_r32) or as floats (out_f32).
int local_grid_rows(int nr);
cudaError_t launch_local_grid(const double *cand, int64_t n_cand, int nr, double gridsize, double *out,
                              double *out_r32, float *out_f32, cudaStream_t s);
cudaError_t launch_block_lists(int64_t n, int64_t per_voxel, int32_t *voxel, int32_t *orient, cudaStream_t s);
// Packed mask back to one byte per pixel (1 = bit set), layout of the distance map.
cudaError_t launch_unpack_bits(const uint32_t *bits, int64_t plane, int64_t nrot, int64_t plane_words, uint8_t *mask,
                               cudaStream_t s);
// Bit-packed hit mask from the 8-bit (or full-width) codes: bit = code < n_hit.
cudaError_t launch_pack_bits(const void *codes, int code_bytes, int64_t plane, int64_t nrot, uint32_t n_hit,
                             int64_t plane_words, uint32_t *bits, cudaStream_t s);
// Enqueue the projection-window sweep over n_trials trials (+ the list refine pass in full mode).
// max_slots (1..64) caps the trials each CTA holds per round (tile height); 0 = 64.  mode as
// launch_scan: kScanFull (8-bit codes, median) or kScanComp (bit-packed mask, counts only, and
// the first maximum per group when b.group_key is set).
cudaError_t launch_sweep(const Geo &g, const ScoreBufs &b, const Work &w, int64_t n_trials, int num_sms,
                         cudaStream_t s, cudaEvent_t ev0, cudaEvent_t ev1, int *launches, int max_slots = 0,
                         int mode = 0);

// Orientation / position preparation kernels.
cudaError_t launch_quat_to_u(const float *q, int64_t n, double *U, cudaStream_t s);
cudaError_t launch_euler_to_u(const float *e, int64_t n, double *U, cudaStream_t s);
cudaError_t launch_f9_to_u(const float *u9, int64_t n, double *U, cudaStream_t s);
cudaError_t launch_pos_f3(const float *p, int64_t n, double *vpos, cudaStream_t s);
cudaError_t launch_pos_rows(const float *rows, int stride, int64_t n, const double *p1, double *vpos,
                            cudaStream_t s);

// Epilogues: TrialRes -> MEX output layouts.
// median false: column 4 is NaN (completeness-only calls).
cudaError_t launch_epi_forward(const TrialRes *res, int64_t n, float *out4, bool median, cudaStream_t s);
// First maximum of completeness per group of gsize consecutive trials (one warp per group) into
// keys (zeroed by the caller; atomicMax of the same keys the completeness scan folds in), and the
// keys decoded into the 0-based index within the group and its completeness.
cudaError_t launch_group_argmax(const TrialRes *res, int64_t n_trials, int64_t gsize, unsigned long long *keys,
                                cudaStream_t s);
cudaError_t launch_group_decode(const unsigned long long *keys, int64_t n_groups, int32_t *best, float *best_c,
                                cudaStream_t s);
cudaError_t launch_epi_grow(const TrialRes *res, const float *rows6, int64_t m, const double *p1, float *out7,
                            cudaStream_t s);
// CSR set-up for compete: counts from rows5 -> items / trial_orient.
cudaError_t launch_csr_counts(const float *rows5, int64_t m, int64_t *counts, cudaStream_t s);
cudaError_t launch_csr_fill(const float *rows5, int64_t m, const int64_t *offsets, const float *id_neigb,
                            int64_t n_neigb, int64_t n_grain, longlong4 *items, int32_t *trial_orient,
                            int32_t *trial_voxel, int *bad, cudaStream_t s);
cudaError_t launch_epi_compete(const TrialRes *res, const longlong4 *items, const int32_t *trial_orient,
                               int64_t m, const float *euler, float *out8, float *trial_out4, cudaStream_t s);

// Device update of the sample maps with compete winners (rows5 1-based indices).
cudaError_t launch_apply_compete(const float *out8, const float *rows5, int64_t m, const int64_t *dims, float *comp,
                                 float *gid, float *dmed, float *ninter, float *visit, cudaStream_t s);

// Distance-map rank coding.
struct MapCodes {
    void *codes;
    uint8_t *codes8;
    float *vals;
    int64_t n_distinct;
    int code_bits;
};
// Encodes d_map (n floats) into codes; allocates codes/vals with cudaMalloc.
cudaError_t encode_map(const float *d_map, int64_t n, cudaStream_t s, MapCodes *out, int *bad_nan);

// Synthetic-data kernels.
cudaError_t launch_simulate_work(const Geo &g, const ScoreBufs &b, const Work &w, int num_sms, uint8_t *mask,
                                 cudaStream_t s);
cudaError_t launch_edt(const uint8_t *mask, int64_t nz, int64_t ny, int64_t nrot, float *map, cudaStream_t s);

// Spot pairing (grc_score.cu: pair_kernel; index built in grc_seed.cu).  Same layout as the
// public grc_spot_pair.
struct PairRec {
    int32_t trial, iw, ih, spot;
    double dety, detz, exp_y, exp_z, area, energy_kev, dis;
};
struct SpotIndex {
    const double *yza;        // 3 per spot: centroid dety, detz [pixel], area [pixel^2]
    const int64_t *cell_off;  // [nrot * ncy * ncz + 1]
    const int32_t *cell_ids;  // spot ids in (projection, cell, list) order
    int ncy, ncz, cell_px;
};
cudaError_t launch_pair(const Geo &g, const ScoreBufs &b, int64_t n, const SpotIndex &si, PairRec *out, int64_t cap,
                        unsigned long long *count, int num_sms, cudaStream_t s);
// Cell index of a spot list: per spot its cell key ((iw * ncy + cy) * ncz + cz), then counts.
cudaError_t launch_spot_keys(const double *yza, const int64_t *proj_off, int nrot, int ncy, int ncz, int cell_px,
                             int32_t *keys, int32_t *ids, int64_t *cell_counts, cudaStream_t s);
cudaError_t launch_pair_keys(const PairRec *p, int64_t n, int nrot, int nhkl, int64_t *keys, int32_t *ids,
                             cudaStream_t s);
cudaError_t launch_pair_gather(const PairRec *in, const int32_t *order, int64_t n, PairRec *out, cudaStream_t s);

// FP64 trial lists (grc_seed.cu): U from double quaternions, work items from (voxel, orientation)
// index pairs (bad |= 1 for an index out of range; that item is left empty).
cudaError_t launch_quat_to_u_d(const double *q, int64_t n, double *U, cudaStream_t s);
// Checks the indices (bad[0] != 0 when one is out of range), builds the work items and sets
// bad[1] to the most voxel-run starts in any aligned block of 32 trials (Work::starts_per_32);
// bad[0..1] must be zero on entry.
cudaError_t launch_trial_items(const int32_t *tv, const int32_t *to, int64_t n, int64_t n_vox, int64_t n_q,
                               longlong4 *items, int *bad, cudaStream_t s);

// Batched bounded Nelder-Mead on 1 - completeness over (q1, q2, q3): one simplex per seed in the
// transformed variables of fminsearchbnd (z), vertices sorted by objective.
struct NmSeed {
    double z[4][3];
    double fv[4];
    double cand[4][3];   // points proposed by the current step
    double lb[3], ub[3];
    int evals, iters, phase, flag;
    int nanmask;         // slots of the current step whose point has no real q0
};
cudaError_t launch_nm_init(NmSeed *st, int64_t n, const double *x0, double half_width, cudaStream_t s);
// Writes U for trials 4i..4i+3 (empty work items for unused slots) and counts running seeds.
cudaError_t launch_nm_propose(NmSeed *st, int64_t n, int max_evals, int max_iter, double tol_f, double tol_x,
                              double *U, longlong4 *items, int *active, cudaStream_t s);
cudaError_t launch_nm_accept(NmSeed *st, int64_t n, const TrialRes *res, cudaStream_t s);
// Loop test of a device-side Nelder-Mead loop (the body of a conditional WHILE graph node): counts
// one more body in *bodies and keeps the loop going while a seed still runs (*active > 0) and
// fewer than max_bodies bodies have run.
cudaError_t launch_nm_continue(unsigned long long handle, const int *active, int *bodies, int max_bodies,
                               cudaStream_t s);
cudaError_t launch_nm_final(const NmSeed *st, int64_t n, double *x, double *fval, int32_t *evals, int32_t *iters,
                            int32_t *flag, cudaStream_t s);

}  // namespace grc
