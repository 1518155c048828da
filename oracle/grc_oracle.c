/*
 * grc_oracle.c -- TEST INFRASTRUCTURE ONLY (the checker, never the product).
 *
 * FP64 CPU restatement of GrainRecon's forward-simulation completeness scorer.
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load this
 * library; the product library (grainrecon_b200/libgrainrecon_b200.so) never
 * links or calls it.
 *
 * Parity status: UNPINNED.  The reference is MATLAB (no MATLAB/Octave on this
 * machine) and its CUDA sources are absent, so no reference output could be
 * produced here and the reference ships no golden vectors.  This file follows
 * the reference line by line instead:
 *   forward_comp.m:4-90                     -> oracle_trial()
 *   ForwardCalc_OR_space_comp.m:22-56       -> oracle_orientation_scan()
 *   quaternion2U.m:3-28, euler2u.m:5-       -> quat_u(), euler_u()
 *   grow_indexed_region_parallel.m:56-88    -> oracle_grow()   (both accept rules)
 *   grow_unindexed_compete_comp_cuda.m:67-94-> oracle_compete()
 * MATLAB semantics kept: round() half away from zero, acos() of a dot product
 * clamped to [-1,1] (the real part of MATLAB's complex result), even-count
 * median = mean of the two middle values, dis_median = 2000 when nothing is
 * simulated, completeness 0/0 = NaN.
 *
 * Inputs use the MEX layouts (float32, matrices row-major as reshape(M',1,9)),
 * promoted to double before any arithmetic.
 *
 * Edge listing: a reflection is an "edge" when its FP64 landing coordinate lies
 * within EDGE_PX of a pixel-rounding boundary, or its wavelength / Bragg angle
 * lies within a relative 1e-9 of a selection threshold.  Every trial reports how
 * many it has.  A "tight edge" uses the bands EDGE_PX_TIGHT (1e-9 px) and
 * EDGE_REL_TIGHT (1e-12): only there can two correct FP64 evaluations of the
 * chain (this acos form and an algebraic form) round differently, so counts of a
 * trial without a tight edge must agree exactly.  The tight count is reported
 * separately (out[4] of oracle_trial, the optional ``tight`` arrays).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define EDGE_PX 1e-4
#define EDGE_REL 1e-9
#define EDGE_PX_TIGHT 1e-9
#define EDGE_REL_TIGHT 1e-12

typedef struct {
    int nhkl, nrot, detysize, detzsize;
    double lss, lsd, p0y, p0z, dety00, detz00, pxy, pxz;
    double bsy0, bsy1, bsz0, bsz1, thetamax, lmin, lmax, rao;
    double dety0, detz0, thr;
    double S[3][3], B[3][3], R[3][3];
    const float *hkl, *map, *rot;
} ogeo;

static void load_m33(double m[3][3], const float *f) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) m[i][j] = (double)f[i * 3 + j];
}

static void geo_init(ogeo *g, const float *S, const float *B, const float *hkl, const float *map,
                     const float *rot, const float *R, const float *param, double dety0, double detz0,
                     double thr) {
    g->nhkl = (int)param[0];
    g->nrot = (int)param[1];
    g->lss = param[2]; g->lsd = param[3]; g->p0y = param[4]; g->p0z = param[5];
    g->dety00 = param[6]; g->detz00 = param[7]; g->pxy = param[8]; g->pxz = param[9];
    g->detysize = (int)param[10]; g->detzsize = (int)param[11];
    g->bsy0 = param[12]; g->bsy1 = param[13]; g->bsz0 = param[14]; g->bsz1 = param[15];
    g->thetamax = param[16]; g->lmin = param[17]; g->lmax = param[18]; g->rao = param[19];
    g->dety0 = dety0; g->detz0 = detz0; g->thr = thr;
    load_m33(g->S, S); load_m33(g->B, B); load_m33(g->R, R);
    g->hkl = hkl; g->map = map; g->rot = rot;
}

static double clamp1(double x) { return x > 1.0 ? 1.0 : (x < -1.0 ? -1.0 : x); }

static int cmp_double(const void *a, const void *b) {
    double x = *(const double *)a, y = *(const double *)b;
    return (x > y) - (x < y);
}

/* MATLAB median: sort, odd -> middle, even -> mean of the two middles. */
static double matlab_median(double *v, int n) {
    if (n == 0) return 2000.0;
    qsort(v, (size_t)n, sizeof(double), cmp_double);
    if (n & 1) return v[n / 2];
    return (v[n / 2 - 1] + v[n / 2]) / 2.0;
}

/* Per-reflection landing record, filled by oracle_landings() for tests. */
typedef struct {
    int32_t iw, ih, sel, edge;
    double u, v, lambda, dis;
} olanding;

/*
 * One (U, pos) trial: forward_comp.m:8-90.  ``dis`` is caller scratch of nrot*nhkl
 * doubles.  Returns out[0..4] = Nr_simu, Nr_intersect, dis_median, the edge count and
 * the tight-edge count; when ``rec`` is non-NULL every reflection's landing record is
 * written there.
 */
static void oracle_trial(const ogeo *g, const double U[3][3], const double pos_in[3], double *dis,
                         double out[4], olanding *rec) {
    const double L = g->lss + g->lsd;
    const double pi = 3.14159265358979323846;
    int nsimu = 0, ninter = 0, nedge = 0, ntight = 0;
    /* Gw = S*U*B*hkl (forward_comp.m:15-16) */
    double SU[3][3], SUB[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            SU[i][j] = 0;
            for (int k = 0; k < 3; ++k) SU[i][j] += g->S[i][k] * U[k][j];
        }
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            SUB[i][j] = 0;
            for (int k = 0; k < 3; ++k) SUB[i][j] += SU[i][k] * g->B[k][j];
        }
    double pos[3] = {pos_in[0], pos_in[1] - g->rao, pos_in[2]}; /* :17 */
    double Spos[3];
    for (int i = 0; i < 3; ++i) Spos[i] = g->S[i][0] * pos[0] + g->S[i][1] * pos[1] + g->S[i][2] * pos[2];
    const double beta_max = (90.0 + g->thetamax * 4.0) / 180.0 * pi;
    const double thr = g->thr;
    for (int iw = 0; iw < g->nrot; ++iw) {
        double omega = (double)g->rot[iw] * pi / 180.0; /* :19 */
        double co = cos(omega), so = sin(omega);
        double SW[3] = {co * Spos[0] - so * Spos[1], so * Spos[0] + co * Spos[1], Spos[2]}; /* :22 */
        double gp[3] = {g->lss + SW[0], SW[1] - g->p0y + g->rao, SW[2] - g->p0z};       /* :26 */
        double center[3] = {L, gp[1] * L / gp[0], gp[2] * L / gp[0]};                  /* :23-24 */
        double alpha = atan(sqrt(gp[1] * gp[1] + gp[2] * gp[2]) / gp[0]);             /* :25 */
        double ngp = sqrt(gp[0] * gp[0] + gp[1] * gp[1] + gp[2] * gp[2]);
        double ncen = sqrt(center[0] * center[0] + center[1] * center[1] + center[2] * center[2]);
        double L2 = (g->lsd - SW[0]) / cos(alpha); /* :42 */
        double dvec[3] = {SW[0] - g->lsd, SW[1] - g->dety00 + g->rao, SW[2] - g->detz00};
        double tnum = g->R[0][0] * (g->lsd - SW[0]) + g->R[1][0] * (g->dety00 - g->rao - SW[1]) +
                      g->R[2][0] * (g->detz00 - SW[2]);
        for (int ih = 0; ih < g->nhkl; ++ih) {
            double h[3] = {g->hkl[3 * ih], g->hkl[3 * ih + 1], g->hkl[3 * ih + 2]};
            double Gw[3];
            for (int i = 0; i < 3; ++i) Gw[i] = SUB[i][0] * h[0] + SUB[i][1] * h[1] + SUB[i][2] * h[2];
            double Gt[3] = {co * Gw[0] - so * Gw[1], so * Gw[0] + co * Gw[1], Gw[2]}; /* :28 */
            double Glen = sqrt(Gt[0] * Gt[0] + Gt[1] * Gt[1] + Gt[2] * Gt[2]);       /* :30 */
            double cb = (gp[0] / ngp) * (Gt[0] / Glen) + (gp[1] / ngp) * (Gt[1] / Glen) +
                        (gp[2] / ngp) * (Gt[2] / Glen);
            double beta = acos(clamp1(cb)); /* :31 */
            double theta = beta - pi / 2;   /* :33 */
            double sintth = sin(2 * theta);
            double d = 1.0 / Glen * 2 * pi;
            double lambda = 2 * d * sin(theta); /* :37 */
            int pass_bl = beta > pi / 2 && beta < beta_max && lambda > g->lmin && lambda < g->lmax;
            int edge = fabs(lambda - g->lmin) <= EDGE_REL * g->lmin ||
                       fabs(lambda - g->lmax) <= EDGE_REL * g->lmax ||
                       fabs(beta - pi / 2) <= EDGE_REL || fabs(beta - beta_max) <= EDGE_REL;
            int tight = fabs(lambda - g->lmin) <= EDGE_REL_TIGHT * g->lmin ||
                        fabs(lambda - g->lmax) <= EDGE_REL_TIGHT * g->lmax ||
                        fabs(beta - pi / 2) <= EDGE_REL_TIGHT || fabs(beta - beta_max) <= EDGE_REL_TIGHT;
            if (!pass_bl && !edge && !rec) continue; /* select3 is a conjunction: skip the rest */
            double konst = sqrt(Gt[1] * Gt[1] + Gt[2] * Gt[2]);                        /* :44 */
            double nv1 = sqrt(0.0 + Gt[1] * Gt[1] + Gt[2] * Gt[2]);
            double cphx = 0.0 * (center[0] / ncen) + (Gt[1] / nv1) * (center[1] / ncen) +
                          (Gt[2] / nv1) * (center[2] / ncen);
            double phix = acos(clamp1(cphx)); /* :40 */
            double phiy = phix - 2 * theta;   /* :41 */
            double diffvec = L2 * sintth / sin(phiy); /* :43 */
            double y22 = center[1] + diffvec * Gt[1] / konst; /* :46 */
            double z22 = center[2] + diffvec * Gt[2] / konst; /* :47 */
            double K[3] = {g->lsd - SW[0], y22 - SW[1], z22 - SW[2]};
            double nK = sqrt((g->lsd - SW[0]) * (g->lsd - SW[0]) + (y22 - SW[1]) * (y22 - SW[1]) +
                             (z22 - SW[2]) * (z22 - SW[2]));
            double Ku[3] = {K[0] / nK, K[1] / nK, K[2] / nK}; /* :49-50 */
            double t = tnum / (g->R[0][0] * Ku[0] + g->R[1][0] * Ku[1] + g->R[2][0] * Ku[2]); /* :51-52 */
            double vv[3] = {t * Ku[0] + dvec[0], t * Ku[1] + dvec[1], t * Ku[2] + dvec[2]};
            double y2 = g->R[0][1] * vv[0] + g->R[1][1] * vv[1] + g->R[2][1] * vv[2]; /* :54 */
            double z2 = g->R[0][2] * vv[0] + g->R[1][2] * vv[1] + g->R[2][2] * vv[2]; /* :55 */
            double u = -y2 / g->pxy + g->dety0, v = -z2 / g->pxz + g->detz0;
            double dety = round(u), detz = round(v); /* :58-59 */
            int sel = pass_bl && dety >= 1 && dety <= g->detysize && detz >= 1 && detz <= g->detzsize &&
                      !(dety >= g->bsy0 && dety <= g->bsy1 && detz >= g->bsz0 && detz <= g->bsz1); /* :61-65 */
            if ((pass_bl || edge) && isfinite(u) && isfinite(v) && u > -2 && v > -2 &&
                u < g->detysize + 3 && v < g->detzsize + 3) {
                double fu = u - floor(u), fv = v - floor(v);
                if (fabs(fu - 0.5) < EDGE_PX || fabs(fv - 0.5) < EDGE_PX) edge = 1;
                if (fabs(fu - 0.5) < EDGE_PX_TIGHT || fabs(fv - 0.5) < EDGE_PX_TIGHT) tight = 1;
            }
            double disv = NAN;
            if (sel) {
                size_t idx = (size_t)(detz - 1) + (size_t)(dety - 1) * (size_t)g->detzsize +
                             (size_t)iw * (size_t)g->detzsize * (size_t)g->detysize;
                disv = (double)g->map[idx]; /* :69 */
                dis[nsimu++] = disv;
                if (disv <= thr) ++ninter; /* :71-72 */
            }
            if (edge) ++nedge;
            if (tight) ++ntight;
            if (rec) {
                olanding *r = &rec[(size_t)iw * g->nhkl + ih];
                r->iw = iw; r->ih = ih; r->sel = sel; r->edge = edge;
                r->u = u; r->v = v; r->lambda = lambda; r->dis = disv;
            }
        }
    }
    out[0] = nsimu;
    out[1] = ninter;
    out[2] = matlab_median(dis, nsimu); /* :86-90 */
    out[3] = nedge;
    out[4] = ntight;
}

static void quat_u(const float *q, double U[3][3]) {
    double q0 = q[0], q1 = q[1], q2 = q[2], q3 = q[3];
    U[0][0] = 2 * (q0 * q0 + q1 * q1) - 1; U[0][1] = 2 * (q1 * q2 - q0 * q3); U[0][2] = 2 * (q1 * q3 + q0 * q2);
    U[1][0] = 2 * (q1 * q2 + q0 * q3); U[1][1] = 2 * (q0 * q0 + q2 * q2) - 1; U[1][2] = 2 * (q2 * q3 - q0 * q1);
    U[2][0] = 2 * (q1 * q3 - q0 * q2); U[2][1] = 2 * (q2 * q3 + q0 * q1); U[2][2] = 2 * (q0 * q0 + q3 * q3) - 1;
}

static void euler_u(double p1, double P, double p2, double U[3][3]) {
    U[0][0] = cos(p1) * cos(p2) - sin(p1) * sin(p2) * cos(P);
    U[1][0] = sin(p1) * cos(p2) + cos(p1) * sin(p2) * cos(P);
    U[2][0] = sin(p2) * sin(P);
    U[0][1] = -cos(p1) * sin(p2) - sin(p1) * cos(p2) * cos(P);
    U[1][1] = -sin(p1) * sin(p2) + cos(p1) * cos(p2) * cos(P);
    U[2][1] = cos(p2) * sin(P);
    U[0][2] = sin(p1) * sin(P);
    U[1][2] = -cos(p1) * sin(P);
    U[2][2] = cos(P);
}

static void pos_from_index(const float *row, const float *p1, double pos[3]) {
    /* grow_indexed_region_parallel.m:70-74; p1 = [RVP(3) simap VoxSize Center(3) Dimension(3) ...] */
    for (int i = 0; i < 3; ++i)
        pos[i] = (((double)row[i] + (double)p1[i] - 1) - (double)p1[8 + i] / 2) * (double)p1[4] + (double)p1[5 + i];
    if (p1[3] == 1.0f) { pos[0] = -pos[0]; pos[1] = -pos[1]; }
}

/* nthreads > 0: use that many threads; otherwise the default the process started with (an earlier
 * call's explicit count does not stick). */
static int default_threads = 0;
static int nthreads_set(int nthreads) {
#ifdef _OPENMP
    if (default_threads == 0) default_threads = omp_get_max_threads();
    omp_set_num_threads(nthreads > 0 ? nthreads : default_threads);
    return omp_get_max_threads();
#else
    (void)nthreads;
    return 1;
#endif
}

/* One trial through the public surface: U row-major (double), pos [mm]; out5 as oracle_trial. */
int oracle_forward_comp(const double *U9, const double *pos, const float *S, const float *B, const float *hkl,
                        const float *map, const float *rot, const float *R, const float *param, double dety0,
                        double detz0, double thr, double *out5) {
    ogeo g;
    geo_init(&g, S, B, hkl, map, rot, R, param, dety0, detz0, thr);
    double U[3][3];
    for (int i = 0; i < 9; ++i) U[i / 3][i % 3] = U9[i];
    double *dis = (double *)malloc(sizeof(double) * (size_t)g.nrot * g.nhkl + 8);
    if (!dis) return -1;
    oracle_trial(&g, U, pos, dis, out5, NULL);
    free(dis);
    return 0;
}

/* Every reflection's landing record for one trial (tests and known-answer cases). */
int oracle_landings(const double *U9, const double *pos, const float *S, const float *B, const float *hkl,
                    const float *map, const float *rot, const float *R, const float *param, double dety0,
                    double detz0, double thr, olanding *rec, double *out5) {
    ogeo g;
    geo_init(&g, S, B, hkl, map, rot, R, param, dety0, detz0, thr);
    double U[3][3];
    for (int i = 0; i < 9; ++i) U[i / 3][i % 3] = U9[i];
    double *dis = (double *)malloc(sizeof(double) * (size_t)g.nrot * g.nhkl + 8);
    if (!dis) return -1;
    oracle_trial(&g, U, pos, dis, out5, rec);
    free(dis);
    return 0;
}

/*
 * ForwardCalc_OR_space_comp.m:22-56 on the cuda_forward_comp argument list:
 * out[4i..4i+3] = [Nr_simu, Nr_intersect, completeness, dis_median] (float),
 * edges[i] = edge-reflection count of orientation i, tight[i] its tight-edge count
 * (either may be NULL).
 */
int oracle_orientation_scan(const float *pos3, const float *q, int64_t n, const float *S, const float *B,
                            const float *hkl, const float *map, const float *rot, const float *R,
                            const float *param, double dety0, double detz0, double thr, int nthreads,
                            float *out, int32_t *edges, int32_t *tight) {
    ogeo g;
    geo_init(&g, S, B, hkl, map, rot, R, param, dety0, detz0, thr);
    double pos[3] = {pos3[0], pos3[1], pos3[2]};
    nthreads_set(nthreads);
    int fail = 0;
#pragma omp parallel
    {
        double *dis = (double *)malloc(sizeof(double) * (size_t)g.nrot * g.nhkl + 8);
        if (!dis) {
#pragma omp atomic write
            fail = 1;
        } else {
#pragma omp for schedule(dynamic, 4)
            for (int64_t i = 0; i < n; ++i) {
                double U[3][3], o[5];
                quat_u(q + 4 * i, U);
                oracle_trial(&g, U, pos, dis, o, NULL);
                out[4 * i] = (float)o[0];
                out[4 * i + 1] = (float)o[1];
                out[4 * i + 2] = (float)(o[1] / o[0]);
                out[4 * i + 3] = (float)o[2];
                if (edges) edges[i] = (int32_t)o[3];
                if (tight) tight[i] = (int32_t)o[4];
            }
            free(dis);
        }
    }
    return fail ? -1 : 0;
}

/*
 * grow_indexed_region_parallel.m:56-88 on the cuda_grow_indexed_region argument
 * list.  rows6 = [x y z I mask DisMedian] (1-based voxel indices), out7 =
 * [x y z Nr_simu Nr_intersect dis_median flag].  rule 0 = the accept rule the
 * GPU kernel can evaluate (no Ninter column is passed), rule 1 = the CPU rule
 * with the |C-I|<=0.01 && Nr_intersect>Ninter clause (needs ``ninter``).
 */
int oracle_grow(const float *rows6, int64_t m, const float *U9f, const float *S, const float *B,
                const float *hkl, const float *map, const float *rot, const float *R, const float *param,
                const float *param1, double dety0, double detz0, double thr, int rule, const float *ninter,
                int nthreads, float *out7, int32_t *edges, int32_t *tight) {
    ogeo g;
    geo_init(&g, S, B, hkl, map, rot, R, param, dety0, detz0, thr);
    double U[3][3];
    for (int i = 0; i < 9; ++i) U[i / 3][i % 3] = (double)U9f[i];
    const double seed_comp = param1[11], drop_off = param1[12], max_dmed = param1[13];
    nthreads_set(nthreads);
    int fail = 0;
#pragma omp parallel
    {
        double *dis = (double *)malloc(sizeof(double) * (size_t)g.nrot * g.nhkl + 8);
        if (!dis) {
#pragma omp atomic write
            fail = 1;
        } else {
#pragma omp for schedule(dynamic, 4)
            for (int64_t i = 0; i < m; ++i) {
                const float *row = rows6 + 6 * i;
                double pos[3], o[5];
                pos_from_index(row, param1, pos);
                oracle_trial(&g, U, pos, dis, o, NULL);
                double C = o[1] / o[0];
                double I = row[3], mask = row[4], dmed = row[5];
                double lim = fmin(dmed, max_dmed);
                int cand = C > I && o[2] <= lim;
                if (rule == 1) cand = cand || (fabs(C - I) <= 0.01 && o[1] > (double)ninter[i]);
                cand = cand && mask > 0;
                int flag = cand && C >= seed_comp * (1 - drop_off);
                float *w = out7 + 7 * i;
                w[0] = row[0]; w[1] = row[1]; w[2] = row[2];
                w[3] = (float)o[0]; w[4] = (float)o[1]; w[5] = (float)o[2]; w[6] = (float)flag;
                if (edges) edges[i] = (int32_t)o[3];
                if (tight) tight[i] = (int32_t)o[4];
            }
            free(dis);
        }
    }
    return fail ? -1 : 0;
}

/*
 * grow_unindexed_compete_comp_cuda.m:44-48 with the argmax of :67-94.
 * rows5 = [x y z first last] (1-based CSR range into id_neigb), id_neigb = grain
 * ids (1-based rows of euler, degrees).  out8 = [i phi1 PHI phi2 GrainId C
 * Nr_intersect dis_median] of the first candidate with the largest completeness
 * (MATLAB max: NaN ignored).  A row with no candidate gives [i 0 0 0 0 0 0 2000].
 */
int oracle_compete(const float *rows5, int64_t m, const float *id_neigb, const float *euler, const float *S,
                   const float *B, const float *hkl, const float *map, const float *rot, const float *R,
                   const float *param, const float *param1, double dety0, double detz0, double thr,
                   int nthreads, float *out8, int32_t *edges, int32_t *tight) {
    ogeo g;
    geo_init(&g, S, B, hkl, map, rot, R, param, dety0, detz0, thr);
    const double pi = 3.14159265358979323846;
    nthreads_set(nthreads);
    int fail = 0;
#pragma omp parallel
    {
        double *dis = (double *)malloc(sizeof(double) * (size_t)g.nrot * g.nhkl + 8);
        if (!dis) {
#pragma omp atomic write
            fail = 1;
        } else {
#pragma omp for schedule(dynamic, 1)
            for (int64_t i = 0; i < m; ++i) {
                const float *row = rows5 + 5 * i;
                double pos[3];
                pos_from_index(row, param1, pos);
                int64_t first = (int64_t)row[3], last = (int64_t)row[4];
                float *w = out8 + 8 * i;
                w[0] = (float)(i + 1);
                for (int k = 1; k < 8; ++k) w[k] = 0;
                w[7] = 2000.0f;
                double bestC = NAN, bestI = 0, bestM = 2000;
                int64_t bestG = -1;
                int ne = 0, nt = 0;
                for (int64_t j = first; j <= last; ++j) {
                    int64_t gid = (int64_t)id_neigb[j - 1];
                    const float *e = euler + 3 * (gid - 1);
                    double U[3][3], o[5];
                    euler_u((double)e[0] * pi / 180, (double)e[1] * pi / 180, (double)e[2] * pi / 180, U);
                    oracle_trial(&g, U, pos, dis, o, NULL);
                    double C = o[1] / o[0];
                    ne += (int)o[3];
                    nt += (int)o[4];
                    if (bestG < 0 || (!isnan(C) && (isnan(bestC) || C > bestC))) {
                        bestC = C; bestI = o[1]; bestM = o[2]; bestG = gid;
                    }
                }
                if (bestG >= 0) {
                    const float *e = euler + 3 * (bestG - 1);
                    w[1] = e[0]; w[2] = e[1]; w[3] = e[2];
                    w[4] = (float)bestG; w[5] = (float)bestC; w[6] = (float)bestI; w[7] = (float)bestM;
                }
                if (edges) edges[i] = ne;
                if (tight) tight[i] = nt;
            }
            free(dis);
        }
    }
    return fail ? -1 : 0;
}

int oracle_max_threads(void) {
#ifdef _OPENMP
    if (default_threads == 0) default_threads = omp_get_max_threads();
    return default_threads;
#else
    return 1;
#endif
}
