/*
 * grainrecon_b200.h -- C ABI of the B200 completeness scorer / grain grower.
 *
 * Drop-in boundary for GrainRecon's CUDA MEX functions.  The three drop-in
 * entries take exactly the arrays the MATLAB wrappers build (float32, matrices
 * flattened row by row as reshape(M',1,9), the distance map flattened
 * column-major as reshape(proj_bin_bw,1,[])) in the same order, and write the
 * same output layout into a caller-owned buffer (host or device memory).
 *
 * Index base: voxel indices in rows6/rows5 and the CSR ranges are 1-based
 * floats, as in the reference.  Every function returns a GRC_* status; no
 * exception or abort crosses this boundary.  The message of the last failure
 * is available from grc_last_error().  One context = one CUDA device + one
 * stream; calls on one context are serialised by an internal mutex.
 */
#ifndef GRAINRECON_B200_H
#define GRAINRECON_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GRC_OK 0
#define GRC_EINVAL 1     /* bad argument (NULL, size, NaN in the map, ...) */
#define GRC_ECAPACITY 2  /* a size beyond a documented limit */
#define GRC_ECUDA 3      /* a CUDA runtime error (message says which) */
#define GRC_ETIMEOUT 4   /* a device-side wait gave up (bounded spin) */
#define GRC_ENOMASK 5    /* no distance map resident and none passed */

/* Documented limits. */
#define GRC_MAX_NHKL 128
#define GRC_MAX_NROT 1800

typedef struct grc_ctx grc_ctx;

/* ---- context ------------------------------------------------------------ */
int grc_ctx_create(grc_ctx **out, int device);
int grc_ctx_destroy(grc_ctx *ctx);
const char *grc_last_error(const grc_ctx *ctx);
/* The context's cudaStream_t (as void*), for callers that enqueue their own work. */
void *grc_ctx_stream(grc_ctx *ctx);
int grc_sync(grc_ctx *ctx);

/*
 * Options the MEX argument list does not carry.  The reference GPU kernels
 * receive neither dety0/detz0 nor minEucDis; the defaults here are the values
 * the reference uses when it re-checks GPU results on the CPU
 * (revise_all_unindexed_voxel_cuda.m:41-42): dety0 = detysize/2+0.5,
 * detz0 = detzsize/2+0.5, hit when dis <= 0.5 pixel.  Pass NaN to keep a default.
 */
int grc_set_options(grc_ctx *ctx, double dety0, double detz0, double hit_threshold_px);

/*
 * Make a distance map resident on the device (replaces the per-call upload of
 * ForwardCalc_OR_space_comp_cuda.m:22 / grow_indexed_region_cuda.m:88).
 * proj_bin_bw: host float32, detzsize*detysize*nrot values, column-major
 * (detz fastest).  The map is rank-coded on the device (16- or 32-bit codes)
 * so the median is exact; NaN values are rejected.
 */
int grc_upload_masks(grc_ctx *ctx, const float *proj_bin_bw, int64_t detzsize, int64_t detysize, int64_t nrot);
/* Same, from device memory (float32, same layout). */
int grc_upload_masks_device(grc_ctx *ctx, const float *d_proj_bin_bw, int64_t detzsize, int64_t detysize,
                            int64_t nrot);

/*
 * Spot masks instead of a distance map: proj_bin holds one byte per pixel (nonzero = spot pixel),
 * detzsize*detysize*nrot bytes in the layout of proj_bin_bw, host or device memory.  The distance
 * map is computed on the device (exact Euclidean distance transform, bwdist semantics: 0 on
 * spot pixels, +Inf for a projection without any) and made resident as by grc_upload_masks.
 * Replaces the host bwdist of GrainMapping_fun.m:73-75 and the per-call upload of the float map.
 */
int grc_upload_spot_masks(grc_ctx *ctx, const uint8_t *proj_bin, int64_t detzsize, int64_t detysize, int64_t nrot);

/*
 * Packed spot-mask files.  grc_save_packed_masks writes the spot pixels (distance 0) of the
 * resident map: an 80-byte header -- magic "GRCMASK1", version 1 (uint32), header size (uint32),
 * detzsize, detysize, nrot, plane_words (int64), the FNV-1a key of the words (uint64), 24
 * reserved bytes -- then nrot * plane_words 32-bit words, plane_words = ceil(detzsize*detysize/128)*4,
 * pixel p = (dety-1)*detzsize + (detz-1) of a projection at bit p&31 of its word p>>5 (little
 * endian).  1 bit per pixel: 189 MB for 361 projections of 2048^2.  grc_load_packed_masks checks
 * the header, the file length and the key (GRC_EINVAL for a truncated, lengthened, altered or
 * foreign file, or a header beyond the map limits of grc_upload_masks, before anything is
 * allocated) and makes the map resident through the device EDT.  (No counterpart in the
 * reference, which keeps the masks in MATLAB .mat files and recomputes bwdist per run.)
 */
int grc_save_packed_masks(grc_ctx *ctx, const char *path);
int grc_load_packed_masks(grc_ctx *ctx, const char *path);

/*
 * Content key of a distance map, for a caller that keeps one map resident across calls: a 64-bit
 * FNV-1a hash of n and of `samples` values spread evenly over the array, first and last
 * included (every value when samples <= 0 or samples >= n); never 0.  MATLAB frees each call's
 * single(reshape(proj_bin_bw,1,[])) temporary (ForwardCalc_OR_space_comp_cuda.m:22), so a later
 * call's array can sit at the same address with other contents: compare keys, not pointers.  A
 * map changed only between sampled positions keeps its key; a caller that edits maps in place
 * uploads with grc_upload_masks.  A host function: no GPU work.  (No counterpart in the
 * reference, which uploads the map on every call.)
 */
uint64_t grc_map_key(const float *proj_bin_bw, int64_t n, int64_t samples);

/*
 * grc_upload_masks when the map's key (grc_map_key with `samples`) or dimensions differ from
 * those of the last upload through this entry; *uploaded (optional) says whether it uploaded.
 * Any other upload (grc_upload_masks*, a drop-in entry with a map) clears the recorded key.
 */
int grc_upload_masks_if_changed(grc_ctx *ctx, const float *proj_bin_bw, int64_t detzsize, int64_t detysize,
                                int64_t nrot, int64_t samples, int *uploaded);

/*
 * Geometry shared by all scorer calls: S, B, RotDet (9 floats, row-major),
 * hkl (3*nhkl floats), rot_angles (nrot floats, degrees) and the 20-float
 * param vector [nhkl nrot Lsam2sou Lsam2det P0y P0z dety00 detz00 pixelysize
 * pixelzsize detysize detzsize BeamStopY(1:2) BeamStopZ(1:2) thetamax
 * lambda_min lambda_max RotAxisOffset] (ForwardCalc_OR_space_comp_cuda.m:25-27).
 */
int grc_set_geometry(grc_ctx *ctx, const float *S, const float *B, const float *hkl, const float *rot_angles,
                     const float *RotDet, const float *param);

/* ---- drop-in entries (host buffers in, caller-owned output) ------------- */

/*
 * Replaces cuda_forward_comp(pos, q, S, B, hkl, proj_bin_bw, rot_angles,
 * RotDet, param) called at ForwardCalc_OR_space_comp_cuda.m:32-33 (also
 * fit_OR_constrain_with_local_comp_cuda.m:47, forward_calc_gridding_OR.m:17).
 * pos: 3 floats [mm]; q: 4*n_q floats [q0 q1 q2 q3] per orientation.
 * out: 4*n_q floats [Nr_simu Nr_intersect completeness dis_median] per
 * orientation (completeness = NaN when Nr_simu = 0; dis_median = 2000 when
 * nothing is simulated).  proj_bin_bw may be NULL when a map is resident;
 * when non-NULL it is uploaded first (the reference's per-call behaviour).
 * No nrot*nhkl capacity limit (the reference stops at 181*80).
 */
int grc_forward_comp(grc_ctx *ctx, const float *pos, const float *q, int64_t n_q, const float *S, const float *B,
                     const float *hkl, const float *proj_bin_bw, const float *rot_angles, const float *RotDet,
                     const float *param, float *out);

/*
 * Replaces cuda_grow_indexed_region(rows6, U, S, B, hkl, proj_bin_bw,
 * rot_angles, RotDet, param, param1) called at grow_indexed_region_cuda.m:105-107
 * and Forward_calc_comp_allvoxel_cuda.m:57-59.
 * rows6: 6*m floats [x y z I mask DisMedian] (x,y,z 1-based voxel indices);
 * U: 9 floats row-major; param1: 14 floats [RecVolumePixel(:,1)'(3) simap
 * VoxSize Center'(3) Dimension(3) seed_comp drop_off maxDmedian].
 * out: 7*m floats [x y z Nr_simu Nr_intersect dis_median growth_flag].  Every
 * row is scored; growth_flag = 1 when mask > 0 and C > I and dis_median <=
 * min(DisMedian, maxDmedian) and C >= seed_comp*(1-drop_off)
 * (grow_indexed_region_parallel.m:78-88 without the Ninter clause, which needs
 * a column the MEX rows do not carry).
 */
int grc_grow_indexed_region(grc_ctx *ctx, const float *rows6, int64_t m, const float *U, const float *S,
                            const float *B, const float *hkl, const float *proj_bin_bw, const float *rot_angles,
                            const float *RotDet, const float *param, const float *param1, float *out);

/*
 * Scores of voxels for a best-first walk: vox holds 3*n 1-based (x, y, z); out receives 3*n
 * doubles [Nr_simu Nr_intersect dis_median].  Returns GRC_OK or an error code that ends the
 * walk.
 */
typedef int (*grc_walk_score_fn)(void *user, const int32_t *vox, int64_t n, double *out);

/*
 * Replaces the region walk of grow_indexed_region.m:32-137 (the CPU path's growth, which the
 * GPU engine uses for spots of at most 2 pixels, GrainMapping_engine_gpu_comp.m), with the
 * scores from `score`.  Maps are X x Y x Z doubles in MATLAB order (x fastest): I
 * (completeness), Imask (> 0 = sample), DisMedian, Ninter; seed: 1-based (x, y, z).  From the
 * current voxel every unvisited in-mask neighbour of the 18 of :50-52 is scored and kept when
 * C > I with dis_median <= min(DisMedian, maxDmedian), or |C - I| <= 0.01 with more
 * intersections than Ninter (:78-79); the walk moves to the first kept voxel of highest C while
 * C / seed_comp > 1 - drop_off.  Out: C_out, D_out, N_out (the input maps with the seed's
 * completeness set to indexed_comp and each grown voxel's values), J_out (1 = grown), idx_out
 * the grown voxels' 1-based linear indices in find() order (*n_idx of them; GRC_ECAPACITY when
 * more than idx_cap, with *n_idx the count needed), center and replace_center of :131-137.
 */
int grc_walk_best_first(grc_walk_score_fn score, void *user, int64_t X, int64_t Y, int64_t Z, const double *I,
                        const double *Imask, const double *DisMedian, const double *Ninter, const int32_t seed[3],
                        double drop_off, double maxD, double indexed_comp, double maxDmedian, double *C_out,
                        double *D_out, double *N_out, uint8_t *J_out, int64_t *idx_out, int64_t idx_cap,
                        int64_t *n_idx, double center[3], int *replace_center);

/*
 * grow_indexed_region.m:1-145 on the GPU scorer: grc_walk_best_first with the voxels scored by
 * the grc_grow_indexed_region kernels for orientation U (9 floats row-major) and the geometry
 * arguments of that entry (param1: its 14 floats; only the first 11, which place voxels, are
 * used).  A voxel's score for one U does not depend on the region, so scores are cached: a
 * request with unscored voxels scores every unscored in-mask voxel of the box reaching 6 voxels
 * beyond them in one kernel call.  proj_bin_bw may be NULL when a map is resident.
 */
int grc_grow_best_first(grc_ctx *ctx, int64_t X, int64_t Y, int64_t Z, const double *I, const double *Imask,
                        const double *DisMedian, const double *Ninter, const int32_t seed[3], double drop_off,
                        double maxD, double indexed_comp, double maxDmedian, const float *U, const float *S,
                        const float *B, const float *hkl, const float *proj_bin_bw, const float *rot_angles,
                        const float *RotDet, const float *param, const float *param1, double *C_out, double *D_out,
                        double *N_out, uint8_t *J_out, int64_t *idx_out, int64_t idx_cap, int64_t *n_idx,
                        double center[3], int *replace_center);

/*
 * Replaces cuda_forward_comp_compete(rows5, id_neigb_all, Euler, S, B, hkl,
 * proj_bin_bw, rot_angles, RotDet, param, param1) called at
 * grow_unindexed_compete_comp_cuda.m:39-41.  rows5: 5*m floats [x y z first
 * last], first/last a 1-based inclusive range into id_neigb (n_neigb floats,
 * 1-based grain ids); euler: 3*n_grain floats (degrees, Bunge ZXZ); param1:
 * the first 11 floats of the grow param1.  out: 8*m floats [row phi1 PHI phi2
 * GrainId completeness Nr_intersect dis_median] of the first candidate with the
 * largest completeness (NaN ignored); a row without candidates gives
 * [row 0 0 0 0 0 0 2000].
 */
int grc_forward_comp_compete(grc_ctx *ctx, const float *rows5, int64_t m, const float *id_neigb, int64_t n_neigb,
                             const float *euler, int64_t n_grain, const float *S, const float *B, const float *hkl,
                             const float *proj_bin_bw, const float *rot_angles, const float *RotDet,
                             const float *param, const float *param1, float *out);

/* ---- device-resident entries (enqueue on the context stream, no sync) --- */

/*
 * Seeding batch: every voxel of d_pos (3*n_vox floats, mm) against every
 * orientation of d_q (4*n_q floats).  d_out: 4*n_vox*n_q floats, voxel-major,
 * same per-trial layout as grc_forward_comp.  Geometry and map must be set.
 */
int grc_forward_comp_device(grc_ctx *ctx, const float *d_pos, int64_t n_vox, const float *d_q, int64_t n_q,
                            float *d_out);

/* Grow on device buffers: d_rows6 (6*m), host U[9] and param1[14], d_out (7*m). */
int grc_grow_device(grc_ctx *ctx, const float *d_rows6, int64_t m, const float *U, const float *param1,
                    float *d_out);

/*
 * Batched grow / compete on a device CSR work list: voxel i (d_rows5 row, 1-based
 * indices) scores candidates id_neigb[first-1 .. last-1] (grain ids into d_euler).
 * d_out: 8*m floats as grc_forward_comp_compete.  When d_trial_out is non-NULL it
 * also receives 4 floats [Nr_simu Nr_intersect C dis_median] per candidate, in
 * CSR order.
 */
int grc_compete_device(grc_ctx *ctx, const float *d_rows5, int64_t m, const float *d_id_neigb, int64_t n_neigb,
                       const float *d_euler, int64_t n_grain, const float *param1, float *d_out,
                       float *d_trial_out);

/*
 * Trial list in FP64 on device buffers: trial t scores voxel d_trial_voxel[t] (a row of
 * d_pos, 3 doubles per voxel [mm]) against orientation d_trial_orient[t] (a row of d_q,
 * 4 doubles [q0 q1 q2 q3] per orientation, used as given).  Both index arrays NULL:
 * trial t = (voxel t, orientation t) and n_vox = n_q = n_trials.  d_out: 4 floats per
 * trial as grc_forward_comp.  This is the scorer called with an FP64 orientation --
 * forward_comp(UU, proj_bin_bw, pos, ...) of GrainMapping_engine_gpu_comp.m:155 and the
 * objective of fit_OR_fun_local.m:2-98 -- batched over any (voxel, orientation) pairs:
 * the local refine grids of fit_OR_constrain_with_local_comp_cuda.m:19-49 (Nr_seed x 730
 * orientations at one voxel) and the final scoring of fitted orientations.  An index out
 * of range is GRC_EINVAL.
 */
int grc_score_trials_device(grc_ctx *ctx, const double *d_pos, int64_t n_vox, const double *d_q, int64_t n_q,
                            const int32_t *d_trial_voxel, const int32_t *d_trial_orient, int64_t n_trials,
                            float *d_out);

/*
 * The same trial list in completeness-only form with the first maximum of every group of
 * group_size consecutive trials (n_trials a multiple of group_size): d_best[g] = 0-based index
 * within group g of its first trial of largest completeness (NaN ignored: MATLAB max), d_best_c[g]
 * that completeness (NaN when every trial of the group is 0/0).  This is the local refine of
 * fit_OR_constrain_with_local_comp_cuda.m:100-110 ([~,ind0] = max(Output(1+nr_per_OR*(j-1):
 * nr_per_OR*j, 3)), one group per candidate grid) and :60 (one group).  d_out (4 floats per trial,
 * column 4 as set by grc_set_median) may be NULL; d_best and d_best_c may be NULL.
 */
int grc_score_trials_argmax_device(grc_ctx *ctx, const double *d_pos, int64_t n_vox, const double *d_q, int64_t n_q,
                                   const int32_t *d_trial_voxel, const int32_t *d_trial_orient, int64_t n_trials,
                                   int64_t group_size, float *d_out, int32_t *d_best, float *d_best_c);

/*
 * Seeding scan with the first maximum over each voxel's orientations: grc_forward_comp_device
 * plus d_best[v] (0-based orientation index of voxel v's first largest completeness, NaN
 * ignored) and d_best_c[v] (that completeness).  d_out may be NULL.
 */
int grc_forward_comp_argmax_device(grc_ctx *ctx, const float *d_pos, int64_t n_vox, const float *d_q, int64_t n_q,
                                   float *d_out, int32_t *d_best, float *d_best_c);

/*
 * Seeding steps 1-2 for n seeds in one call (GrainMapping_engine_gpu_comp.m:72-111): the
 * completeness-only scan of every seed (d_pos: 3 floats per seed [mm]) against the n_q
 * orientations of d_q (4 floats [q0 q1 q2 q3] each, as the MEX receives them), then per seed the
 * first n_top rows of sortrows(Output, 3, 'descend') -- NaN first, larger completeness next, equal
 * values in grid order.  d_idx (n*n_top int32): 0-based rows of d_q, best first; d_cand (optional,
 * n*n_top*4 doubles): those rows, taken from d_q64 (the same orientations in double, optional) or
 * else widened from d_q; d_out (optional, 4*n*n_q floats): the scan, column 4 NaN.
 * 1 <= n_top <= min(4096, n_q).
 */
int grc_seed_candidates_device(grc_ctx *ctx, const float *d_pos, int64_t n, const float *d_q, const double *d_q64,
                               int64_t n_q, int n_top, int32_t *d_idx, double *d_cand, float *d_out);

/*
 * Seeding step 3 for n seeds with k candidates each (fit_OR_constrain_with_local_comp_cuda.m:12-49,
 * 100-116): every candidate's ori_local_sampling(q, nr, gridsize) grid ((nr+1)^3 + 1 rows in
 * unique(q,'rows') order, scored rounded to float32 as the MEX receives them) at its seed, in
 * completeness-only mode, and the first maximum of each grid; then per seed the candidates in
 * sortrows(Output_max, 3, 'descend') order.  d_pos: 3 doubles per seed; d_cand: n*k*4 doubles.
 * Out, per seed in that order: d_best_q (n*k*4 doubles, the FP64 grid row of each maximum),
 * d_best_c (n*k floats, its completeness), d_order (n*k int32, the 0-based candidate it came
 * from), and optionally d_x0 (n*n_x0*3 doubles: [b c d] of the first n_x0 rows, the start points
 * of the orientation fit, :116).  At most 1024 grid rows (nr <= 9) and 4096 candidates per seed.
 */
int grc_seed_refine_device(grc_ctx *ctx, const double *d_pos, int64_t n, const double *d_cand, int k, int nr,
                           double gridsize, int n_x0, double *d_best_q, float *d_best_c, int32_t *d_order,
                           double *d_x0);

/*
 * ori_local_sampling(q, nr, gridsize) (ori_local_sampling.m:12-34) of n_cand quaternions (4 doubles
 * each): (nr+1)^3 + 1 rows per candidate [sqrt(1-(b^2+c^2+d^2)) b c d] with the centre row, in
 * unique(q,'rows') order (a row equal to another stays beside it), into d_rows (doubles) and
 * optionally d_rows_f32 (the same rows rounded to float32).  nr <= 9.
 */
int grc_local_grid_device(grc_ctx *ctx, const double *d_cand, int64_t n_cand, int nr, double gridsize,
                          double *d_rows, float *d_rows_f32);

/*
 * Median of the seeding-scan entries (grc_forward_comp, grc_forward_comp_device,
 * grc_score_trials_device and the two argmax forms above).  1 (default): the reference's four
 * columns, dis_median exact.  0: completeness only -- column 4 is NaN and Nr_simu, Nr_intersect
 * come from a bit-packed hit mask (1 bit per pixel: distance <= the hit threshold), which the
 * context builds on the device from its resident map when first needed.  The seeding engine reads
 * column 3 only: GrainMapping_engine_gpu_comp.m:103 sorts the scan on it and
 * fit_OR_constrain_with_local_comp_cuda.m:60,105 take its maximum.  Grow and compete always
 * compute the median (their accept rule reads it), and so does grc_forward_comp_noalloc.
 */
int grc_set_median(grc_ctx *ctx, int enable);

/*
 * Batched orientation fit of the seeding stage: for each of n seeds, a bounded
 * Nelder-Mead (fminsearchbnd over (q1, q2, q3), bounds max(x0-hw,-1)..min(x0+hw,1),
 * q0 = sqrt(1 - q1^2 - q2^2 - q3^2)) minimising 1 - completeness at the seed position.
 * Replaces the per-seed fminsearchbnd(fit_OR_fun_local, ...) call of
 * fit_OR_constrain_with_local_comp_cuda.m:115-126 (hw 0.02, MaxFunEvals = MaxIter = 2000,
 * TolFun 1e-10, TolX 1e-4 in fminsearch's default).  Every simplex follows the sequential
 * fminsearch rules (reflection 1, expansion 2, contractions 1/2, shrink 1/2, initial
 * simplex x0 and 5% steps, the 2*pi shift of the sine transform); all seeds advance
 * together, one scorer launch per step.  d_pos: 3 doubles per seed [mm]; d_x0: 3 doubles
 * per seed.  Outputs (device): d_x (3 per seed, the fitted q1..q3), d_fval (1 - C at d_x's
 * simplex vertex), and optionally d_evals, d_iters, d_flag (int32: 1 converged by
 * TolFun/TolX, 0 stopped by MaxFunEvals/MaxIter).  Returns after the work has finished.
 */
int grc_fit_orientation_nm(grc_ctx *ctx, const double *d_pos, const double *d_x0, int64_t n, double half_width,
                           int max_evals, int max_iter, double tol_f, double tol_x, double *d_x, double *d_fval,
                           int32_t *d_evals, int32_t *d_iters, int32_t *d_flag);

/*
 * Spot pairing of forward_comp_pair_spots.m:60-85 (called by the orientation fit,
 * fit_OR_constrain_with_local_comp_cuda.m:150-153, and the grain-centre fit): for every trial
 * (FP64 position, quaternion as grc_score_trials_device) and every selected reflection whose
 * pixel is a hit, the nearest measured spot centroid of that projection is paired when it lies
 * closer than min(sqrt(area), 15) pixels (the first spot in list order among equal distances).
 * d_spots: 3 doubles per spot [dety centroid, detz centroid, area] (Spots{i}(:,9:11)), the spots
 * of projection i (0-based) at [d_proj_offsets[i], d_proj_offsets[i+1]) (nrot+1 int64 values).
 * d_pairs receives the pairs in the reference's order (trial, projection, reflection);
 * *n_pairs the number found.  More than max_pairs is GRC_ECAPACITY with *n_pairs set to the
 * number needed.  Returns after the work has finished.
 */
typedef struct grc_spot_pair {
    int32_t trial;      /* 0-based trial */
    int32_t iw;         /* 0-based projection */
    int32_t ih;         /* 0-based reflection (row of hkl) */
    int32_t spot;       /* 0-based index into d_spots */
    double dety, detz;  /* simulated pixel, 1-based (dety, detz of forward_comp.m:58-59) */
    double exp_y, exp_z;/* the paired centroid */
    double area;        /* its area [pixel^2] */
    double energy_kev;  /* 12.398 / lambda of the reflection */
    double dis;         /* distance-map value at the simulated pixel */
} grc_spot_pair;
int grc_pair_spots(grc_ctx *ctx, const double *d_pos, const double *d_q, int64_t n, const double *d_spots,
                   int64_t n_spots, const int64_t *d_proj_offsets, grc_spot_pair *d_pairs, int64_t max_pairs,
                   int64_t *n_pairs);

/*
 * Allocation-free seeding scan (no counterpart in the reference: the MEX functions
 * always allocate their gpuArray output).  For callers that must not allocate GPU
 * memory while they score -- a MEX shim inside MATLAB's gpuArray memory manager, a
 * framework whose caching allocator owns the device, a per-seed loop where cudaMalloc
 * or cudaFree would synchronise the device.  Same results as grc_forward_comp for one
 * voxel: pos is 3 host floats [mm]; d_q (4*n_q floats) and d_out (4*n_q floats) are
 * caller-owned device buffers.  Geometry and distance map must already be resident
 * (set up earlier with grc_set_geometry / grc_upload_masks).
 *
 * Its scratch is one fixed device array of about 6.3 MB, compiled into the library and
 * held by every GPU that loads it until the process exits; n_q above
 * GRC_NOALLOC_MAX_ORIENTATIONS is rejected with GRC_ECAPACITY.  The first call on a
 * device looks up that array's device address (cudaGetSymbolAddress), so make that
 * first call before any stream capture.  All calls in the process share the array and
 * each call leaves its contents behind: calls that overlap on the GPU (from different
 * contexts or threads on the same device) race and must be serialised by the caller.
 * The call returns after its work has finished on the context stream.
 */
#define GRC_NOALLOC_MAX_ORIENTATIONS 65536
int grc_forward_comp_noalloc(grc_ctx *ctx, const float *pos, const float *d_q, int64_t n_q, float *d_out);

/*
 * Batched grower (uneven candidate sets; the grow iteration of
 * grow_unindexed_compete_comp_cuda.m:3-65 / revise_all_unindexed_voxel_cuda.m).
 * grc_batch_create builds the CSR work list of a fixed voxel set once (device rows5,
 * id_neigb, euler, as grc_compete_device; they must stay valid while the batch lives) and
 * binds it to the context's current geometry and map, which must not change while the
 * batch lives.  grc_batch_run enqueues one iteration (scoring of every candidate, the
 * per-voxel argmax into d_out8, and the optional map update) with no host
 * synchronisation; grc_batch_capture records that sequence into a CUDA graph that
 * grc_batch_replay launches.  grc_batch_autotune times the scoring tile shapes
 * (per-trial kernel, or the CTA sweep or warp scan holding 16/32/48/64 trials per CTA)
 * on the first max_voxels voxels, keeps the fastest for this batch and caches it per
 * geometry for later batches.  grc_batch_set_maps makes every run also write each
 * voxel's completeness, grain id, dis_median, Nr_intersect and VisitFlag = 0.5 into
 * device volumes (float, dims[0] x dims[1] x dims[2], column-major, any may be NULL).
 */
typedef struct grc_batch grc_batch;
int grc_batch_create(grc_ctx *ctx, const float *d_rows5, int64_t m, const float *d_id_neigb, int64_t n_neigb,
                     const float *d_euler, int64_t n_grain, const float *param1, grc_batch **out);
int grc_batch_set_maps(grc_batch *batch, const int64_t *dims, float *d_completeness, float *d_grain_id,
                       float *d_dismedian, float *d_ninter, float *d_visitflag);
int grc_batch_run(grc_batch *batch, float *d_out8, float *d_trial_out);
int grc_batch_capture(grc_batch *batch, float *d_out8);
int grc_batch_replay(grc_batch *batch);
int grc_batch_autotune(grc_batch *batch, float *d_out8, int64_t max_voxels, int *path, int *slots, double *best_ms);
int grc_batch_info(grc_batch *batch, int64_t *n_voxels, int64_t *n_trials, int *path, int *slots);
int grc_batch_destroy(grc_batch *batch);

/*
 * Spot-centroid fits (replace fminsearchbnd in fit_OR_constrain_* / fit_grain_COM.m and
 * GrainMapping_fit_geo.m / L_shift_tilt_fitting.m).  The residual of a matched spot is the
 * continuous landing point (u, v) [pixel] of forward_comp.m:28-59 (no rounding) minus the
 * measured centroid.  Fixed geometry (S, B, hkl, rot_angles, pixel sizes, detector size,
 * beam centre, wavelength window) comes from grc_set_geometry / grc_set_options; the fitted
 * quantities are doubles:
 *   grain  (6 per grain): Rodrigues vector r (U from q0 = 1/sqrt(1+|r|^2), q = r q0), centre [mm]
 *   geo10: Lsam2sou, Lsam2det, dety00, detz00, tilt_x, tilt_y, tilt_z [deg] (RotDet = Rz*Ry*Rx,
 *          get_det_R.m:1-7), P0y, P0z, RotAxisOffset.
 * Spots: d_grain (0-based grain index), d_iw (omega index), d_ih (hkl index) int32, d_uv
 * (2 doubles, measured centroid); for per-grain fits the spots of a grain are contiguous and
 * d_offsets (n_grains+1) delimits them.  All pointers named d_* are device memory.
 */
/* Synthetic matched spots: count / fill the selected landings of each grain (no noise). */
int grc_fit_spot_count(grc_ctx *ctx, const double *geo10, const double *d_grains, int64_t n_grains,
                       int64_t *d_counts);
int grc_fit_spot_fill(grc_ctx *ctx, const double *geo10, const double *d_grains, int64_t n_grains,
                      const int64_t *d_offsets, int32_t *d_grain, int32_t *d_iw, int32_t *d_ih, double *d_uv);
/*
 * Residuals (model - measured, 2 per spot) and Jacobian rows d(u,v)/d(params) (2*K per
 * spot, u row then v row) by hand-propagated FP64 tangents; mode 0: K = 6 grain parameters,
 * mode 1: K = 10 geometry parameters.  The loss gradient is J^T r.  A spot that leaves the
 * wavelength window or the detector gets NaN residuals.
 */
int grc_centroid_residual_adjoint(grc_ctx *ctx, int mode, const double *geo10, const double *d_grains,
                                  const int32_t *d_grain, const int32_t *d_iw, const int32_t *d_ih,
                                  const double *d_uv, int64_t n_spots, double *d_res, double *d_jac);
/* Levenberg-Marquardt on every grain (6x6 FP64 normal equations per grain), `iters` iterations
 * or until no grain improves; d_lambda (one damping value per grain) carries over calls. */
int grc_fit_grains_lm(grc_ctx *ctx, const double *geo10, double *d_grains, int64_t n_grains, const int32_t *d_grain,
                      const int32_t *d_iw, const int32_t *d_ih, const double *d_uv, int64_t n_spots,
                      const int64_t *d_offsets, double *d_lambda, int iters, int *n_improved);
/* Forward-only baseline: batched Nelder-Mead with fminsearchbnd's sine bound transform
 * (fminsearchbnd.m:263-265) inside [start - half_width, start + half_width]; d_trace (optional)
 * receives the best point every `checkpoint` evaluations (n_ck x n_grains x 6). */
int grc_fit_grains_nm(grc_ctx *ctx, const double *geo10, double *d_grains, int64_t n_grains, const int32_t *d_grain,
                      const int32_t *d_iw, const int32_t *d_ih, const double *d_uv, int64_t n_spots,
                      const int64_t *d_offsets, const double *half_width, int max_evals, int checkpoint,
                      double *d_trace, int n_ck);
/* Per-grain RMS distance [pixel] of the predicted spots of d_grains from those of d_truth. */
int grc_fit_grains_rms(grc_ctx *ctx, const double *geo10, const double *d_grains, const double *d_truth,
                       int64_t n_grains, const int32_t *d_grain, const int32_t *d_iw, const int32_t *d_ih,
                       const double *d_uv, int64_t n_spots, const int64_t *d_offsets, double *d_rms);
/* Levenberg-Marquardt on the 10 geometry parameters of n_starts starting points at once (10x10
 * FP64 normal equations reduced over all spots per start); grains held fixed. */
int grc_fit_geometry_lm(grc_ctx *ctx, double *d_starts, int n_starts, const double *d_grains, const int32_t *d_grain,
                        const int32_t *d_iw, const int32_t *d_ih, const double *d_uv, int64_t n_spots,
                        double *d_lambda, int iters, int *n_improved);
/* Sum of squared residuals and spot count (2 doubles) of each geometry point (forward only). */
int grc_fit_geometry_cost(grc_ctx *ctx, const double *d_points, int n_points, const double *d_grains,
                          const int32_t *d_grain, const int32_t *d_iw, const int32_t *d_ih, const double *d_uv,
                          int64_t n_spots, double *d_cost);
/* Sum of squared distances and count (2 doubles per start) of predicted spots from those of the
 * geometry geo_truth10 (host). */
int grc_fit_geometry_rms(grc_ctx *ctx, const double *d_starts, int n_starts, const double *geo_truth10,
                         const double *d_grains, const int32_t *d_grain, const int32_t *d_iw, const int32_t *d_ih,
                         const double *d_uv, int64_t n_spots, double *d_acc);

/* Statistics of the last scorer launch on this context. */
typedef struct {
    int64_t trials;          /* (voxel, orientation) pairs scored */
    int64_t refined;         /* trials whose median needed the exact refine pass */
    int64_t kernel_launches; /* kernels enqueued by the call */
    double score_ms;         /* device time of the scoring kernel(s) (CUDA events), 0 if not timed */
    int64_t path;            /* 1 = per-trial kernel, 2 = CTA sweep, 3 = warp scan */
    int64_t audit_checked;   /* audit builds only: FP32 decisions re-decided in FP64 */
    int64_t audit_mismatch;  /* audit builds only: of those, decisions that differed */
    int64_t device_loop;     /* grc_fit_orientation_nm: 1 when its iterations ran as one graph whose
                                conditional WHILE node stops on the device, 0 when the host replayed
                                the steps */
} grc_stats;
int grc_last_stats(grc_ctx *ctx, grc_stats *out);
/* 1 = record CUDA events around the scoring kernel of each call (for benchmarks). */
int grc_set_timing(grc_ctx *ctx, int enable);
/*
 * Scoring kernel selection: 0 = by size (default: the projection-window warp scan, which keeps
 * the map windows L2-resident and runs one trial per warp at a time, once a call holds 1/16 of a
 * round of trials -- 1,776 on 148 SMs -- when each voxel carries at least 64 orientations, or
 * half a round otherwise; the CTA sweep for full-output calls of more than two rounds; the
 * per-trial kernel below that), 1 = always the per-trial kernel,
 * 2 = always the CTA sweep (the same windows with the trials of a CTA mixed in its batches),
 * 3 = always the warp scan.  Results are identical; only speed differs.  Batches (grc_batch_*)
 * read the same codes for their tile choice.
 */
int grc_set_path(grc_ctx *ctx, int path);

/* Counts of selected reflections per trial are exact; this reports the codes of the
 * resident map: number of distinct values, code width in bits. */
int grc_mask_info(grc_ctx *ctx, int64_t *n_distinct, int *code_bits, int64_t *detzsize, int64_t *detysize,
                  int64_t *nrot);

/*
 * Synthetic-data helpers (device-side mask preparation).
 * grc_simulate_spots: every voxel (d_pos, 3*n floats mm) with its orientation
 * (d_U, 9*n floats row-major) lands its selected reflections; the landing
 * pixels are OR-ed into d_mask (uint8, nrot*detysize*detzsize, detz fastest).
 * grc_edt: exact Euclidean distance transform per projection (bwdist
 * semantics: distance to the nearest nonzero mask pixel, +Inf for a projection
 * with none) into d_map (float32, same layout).
 */
int grc_simulate_spots(grc_ctx *ctx, const float *d_pos, const float *d_U, int64_t n, uint8_t *d_mask);
int grc_edt(grc_ctx *ctx, const uint8_t *d_mask, int64_t detzsize, int64_t detysize, int64_t nrot, float *d_map);

#ifdef __cplusplus
}
#endif
#endif
