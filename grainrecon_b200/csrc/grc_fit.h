// grc_fit.h -- types and launchers of the spot-centroid fits (grc_fit.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace grc {

// Geometry that stays fixed during a fit (from the context's geometry and options).
struct FitFixed {
    double S[9], B[9];
    double pxy, pxz, dety0, detz0, lmin, lmax, cbmax;
    int detysize, detzsize, nrot, nhkl;
    const double2 *rot_cs;
    const double *hkl;
};

// Matched spots: grain index, omega index, hkl index, measured (u, v) centroid [pixel].
// Spots of one grain are contiguous when offsets are used.
struct SpotList {
    int32_t *grain;
    int32_t *iw;
    int32_t *ih;
    double *uv;
    int64_t n;
};

cudaError_t fit_residual_jacobian(const FitFixed &fx, int mode, const double *grains, const double *geo10,
                                  const SpotList &sp, double *res, double *jac, cudaStream_t s);
cudaError_t fit_spots_count(const FitFixed &fx, const double *grains, const double *geo10, int64_t n_grains,
                            int64_t *counts, cudaStream_t s);
cudaError_t fit_spots_fill(const FitFixed &fx, const double *grains, const double *geo10, int64_t n_grains,
                           const int64_t *offsets, const SpotList &sp, cudaStream_t s);
cudaError_t fit_grain_normal(const FitFixed &fx, const double *grains, const double *geo10, const SpotList &sp,
                             const int64_t *offsets, int64_t n_grains, double *ne, cudaStream_t s);
cudaError_t fit_grain_cost(const FitFixed &fx, const double *grains, const double *geo10, const SpotList &sp,
                           const int64_t *offsets, int64_t n_grains, double *cost, cudaStream_t s);
cudaError_t fit_grain_rms(const FitFixed &fx, const double *grains, const double *truth, const double *geo10,
                          const SpotList &sp, const int64_t *offsets, int64_t n_grains, double *rms, cudaStream_t s);
cudaError_t fit_grain_lm_propose(const double *grains, const double *ne, const double *lambda, int64_t n,
                                 double *trial, cudaStream_t s);
cudaError_t fit_grain_lm_accept(double *grains, const double *trial, const double *cost_now, const double *cost_trial,
                                double *lambda, int64_t n, int *improved, cudaStream_t s);
cudaError_t fit_grain_nm(const FitFixed &fx, double *grains, const double *geo10, const SpotList &sp,
                         const int64_t *offsets, int64_t n_grains, const double *half_width, int max_evals,
                         int checkpoint, double *trace, int n_ck, cudaStream_t s);
cudaError_t fit_geo_normal(const FitFixed &fx, const double *grains, const double *starts, int n_starts,
                           const SpotList &sp, double *ne, int num_sms, cudaStream_t s);
cudaError_t fit_geo_cost(const FitFixed &fx, const double *grains, const double *starts, int n_starts,
                         const SpotList &sp, double *cost, int num_sms, cudaStream_t s);
cudaError_t fit_geo_rms(const FitFixed &fx, const double *grains, const double *starts, int n_starts,
                        const double *truth, const SpotList &sp, double *acc, int num_sms, cudaStream_t s);
cudaError_t fit_geo_lm_propose(const double *starts, const double *ne, const double *lambda, int n, double *trial,
                               cudaStream_t s);
cudaError_t fit_geo_lm_accept(double *starts, const double *trial, const double *cost_now, const double *cost_trial,
                              double *lambda, int n, int *improved, cudaStream_t s);

}  // namespace grc
