/*
 * grc_synth_host.c -- TEST AND BENCHMARK INFRASTRUCTURE ONLY (never the product).
 *
 * Host-side synthesis of the benchmark inputs, so that the CPU reference arm of the
 * benchmark builds its sample and distance map without a GPU and without the product
 * library:
 *   host_power_voronoi  -- grain ids of a cylinder split by a power diagram (the same
 *                          sites, weights and arithmetic order as the numpy generator
 *                          grainrecon_b200.synth.voronoi_cylinder);
 *   host_simulate_mask  -- spot masks: every voxel lands its selected reflections with its
 *                          grain's orientation (forward_comp.m:15-65 in the algebraic FP64
 *                          form the product's synthesiser uses: sin(theta) = -cos(beta),
 *                          ray/plane intersection without normalising the ray);
 *   host_edt            -- bwdist per projection (GrainMapping_fun.m:73-75): exact Euclidean
 *                          distance from every pixel to the nearest spot pixel, +Inf for a
 *                          projection with none, by the two-pass lower-envelope method of
 *                          Felzenszwalb and Huttenlocher (2012).
 * Layouts: volumes C-order (x slowest); masks and maps (nrot, dety, detz), detz fastest
 * (the MATLAB detz x dety x nrot array flattened by reshape(proj_bin_bw,1,[])).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* Threads of one parallel region: n > 0, else the OpenMP default. */
static int pick_threads(int n) {
#ifdef _OPENMP
    return n > 0 ? n : omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}

/* gid[(ix*dim + iy)*dim + iz] = 1 + argmin_j (|p - s_j|^2 - w2_j) inside the cylinder
 * (x - r)^2 + (y - r)^2 <= r^2 (r = dim/2, p = index + 0.5), else 0.  The squared
 * distance is summed x, y, z in that order, as numpy's sum over a 3-vector. */
int host_power_voronoi(int dim, const double *sites, const double *w2, int n_sites, int nthreads,
                       int32_t *gid) {
    if (dim < 1 || n_sites < 1) return -1;
    const int nt = pick_threads(nthreads);
    const double r = dim / 2.0;
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
    for (int ix = 0; ix < dim; ++ix) {
        const double x = ix + 0.5;
        for (int iy = 0; iy < dim; ++iy) {
            const double y = iy + 0.5;
            const int inside = (x - r) * (x - r) + (y - r) * (y - r) <= r * r;
            for (int iz = 0; iz < dim; ++iz) {
                const double z = iz + 0.5;
                int32_t best = 0;
                if (inside) {
                    double bd = INFINITY;
                    for (int j = 0; j < n_sites; ++j) {
                        const double dx = x - sites[3 * j], dy = y - sites[3 * j + 1], dz = z - sites[3 * j + 2];
                        const double d = ((dx * dx + dy * dy) + dz * dz) - w2[j];
                        if (d < bd) {
                            bd = d;
                            best = j + 1;
                        }
                    }
                }
                gid[((int64_t)ix * dim + iy) * dim + iz] = best;
            }
        }
    }
    return 0;
}

/*
 * Spot masks of n voxels: voxel i at pos[3i..3i+2] [mm] with orientation Ugrain[9*(gid[i]-1)]
 * (row-major).  Geometry in the MEX layouts (float32 S, B, RotDet row-major, hkl 3 per
 * reflection, rot_angles in degrees, the 20-float param).  Selected landing pixels are set to
 * 1 in mask (nrot x detysize x detzsize bytes).
 */
int host_simulate_mask(const float *Sf, const float *Bf, const float *hklf, const float *rot, const float *Rf,
                       const float *param, double dety0, double detz0, const double *pos, const int32_t *gid,
                       int64_t n, const double *Ugrain, int64_t n_grain, int nthreads, uint8_t *mask) {
    const int nhkl = (int)param[0], nrot = (int)param[1];
    const double lss = param[2], lsd = param[3], p0y = param[4], p0z = param[5];
    const double y00 = param[6], z00 = param[7], pxy = param[8], pxz = param[9];
    const int ny = (int)param[10], nz = (int)param[11];
    const double bsy0 = param[12], bsy1 = param[13], bsz0 = param[14], bsz1 = param[15];
    const double tmax = param[16], lmin = param[17], lmax = param[18], rao = param[19];
    const double pi = 3.14159265358979323846;
    const double bmax = (90.0 + 4.0 * tmax) / 180.0 * pi;
    const double cbmax = bmax <= pi ? cos(bmax) : -2.0;
    double S[9], B[9], R[9];
    for (int i = 0; i < 9; ++i) {
        S[i] = Sf[i];
        B[i] = Bf[i];
        R[i] = Rf[i];
    }
    double *cs = (double *)malloc(sizeof(double) * 2 * nrot);
    double *SUBh = (double *)malloc(sizeof(double) * 6 * nhkl * n_grain);
    if (!cs || !SUBh) {
        free(cs);
        free(SUBh);
        return -1;
    }
    for (int iw = 0; iw < nrot; ++iw) {
        const double w = (double)rot[iw] * pi / 180.0;
        cs[2 * iw] = cos(w);
        cs[2 * iw + 1] = sin(w);
    }
    /* Gw = S*U*B*h and |Gw| per grain and reflection, plus the window on t = -(k_w . Gw) =
     * |Gw| lambda / (4 pi) * |Gw| widened by a margin far above its rounding: a reflection outside
     * it cannot pass the exact test below, which decides every reflection inside it */
    for (int64_t gi = 0; gi < n_grain; ++gi) {
        const double *U = Ugrain + 9 * gi;
        double SU[9], SUB[9];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                SU[3 * i + j] = S[3 * i] * U[j] + S[3 * i + 1] * U[3 + j] + S[3 * i + 2] * U[6 + j];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                SUB[3 * i + j] = SU[3 * i] * B[j] + SU[3 * i + 1] * B[3 + j] + SU[3 * i + 2] * B[6 + j];
        for (int ih = 0; ih < nhkl; ++ih) {
            const double h = hklf[3 * ih], k = hklf[3 * ih + 1], l = hklf[3 * ih + 2];
            double *o = SUBh + 6 * ((int64_t)gi * nhkl + ih);
            o[0] = SUB[0] * h + SUB[1] * k + SUB[2] * l;
            o[1] = SUB[3] * h + SUB[4] * k + SUB[5] * l;
            o[2] = SUB[6] * h + SUB[7] * k + SUB[8] * l;
            o[3] = sqrt(o[0] * o[0] + o[1] * o[1] + o[2] * o[2]);
            const double G2 = o[3] * o[3], m = 1e-9 * o[3];
            double hi = lmax * G2 / (4.0 * pi);
            if (cbmax > -1.0 && -cbmax * o[3] < hi) hi = -cbmax * o[3];
            o[4] = lmin * G2 / (4.0 * pi) - m;
            o[5] = hi + m;
        }
    }
    const int64_t plane = (int64_t)ny * nz;
    const double L = lss + lsd;
    const int nt = pick_threads(nthreads);
    int bad = 0;
#pragma omp parallel for schedule(dynamic, 64) num_threads(nt)
    for (int64_t i = 0; i < n; ++i) {
        const int64_t g = (int64_t)gid[i] - 1;
        if (g < 0 || g >= n_grain) {
#pragma omp atomic write
            bad = 1;
            continue;
        }
        const double px = pos[3 * i], py = pos[3 * i + 1] - rao, pz = pos[3 * i + 2];
        const double spx = S[0] * px + S[1] * py + S[2] * pz;
        const double spy = S[3] * px + S[4] * py + S[5] * pz;
        const double spz = S[6] * px + S[7] * py + S[8] * pz;
        const double *gw = SUBh + 6 * g * nhkl;
        for (int iw = 0; iw < nrot; ++iw) {
            const double c = cs[2 * iw], s = cs[2 * iw + 1];
            const double swx = c * spx - s * spy, swy = s * spx + c * spy, swz = spz;
            const double gx = lss + swx, gy = swy - p0y + rao, gz = swz - p0z;
            const double ngp = sqrt(gx * gx + gy * gy + gz * gz);
            const double kx = gx / ngp, ky = gy / ngp, kz = gz / ngp;
            const double L2 = (lsd - swx) * ngp / gx;
            const double ax = lsd - swx, ay = gy * L / gx - swy, az = gz * L / gx - swz;
            const double dx = swx - lsd, dy = swy - y00 + rao, dz = swz - z00;
            const double num = -(R[0] * dx + R[3] * dy + R[6] * dz);
            const double r2d = R[1] * dx + R[4] * dy + R[7] * dz;
            const double r3d = R[2] * dx + R[5] * dy + R[8] * dz;
            /* k_w = Omega^T k: k . (Omega Gw) = k_w . Gw */
            const double wx = c * kx + s * ky, wy = -s * kx + c * ky, wz = kz;
            for (int ih = 0; ih < nhkl; ++ih) {
                const double *G = gw + 6 * ih;
                const double t = -(wx * G[0] + wy * G[1] + wz * G[2]);
                if (!(t > G[4] && t < G[5])) continue;
                const double x = -t / G[3]; /* cos(beta) */
                const double lam = 2.0 * (2.0 * pi / G[3]) * (-x);
                if (!(x < 0.0 && x > cbmax && lam > lmin && lam < lmax)) continue;
                const double Gty = s * G[0] + c * G[1], Gtz = G[2];
                const double st = -x, ct = sqrt(1.0 - x * x);
                const double s2 = 2.0 * st * ct, c2 = 1.0 - 2.0 * st * st;
                const double konst = sqrt(Gty * Gty + Gtz * Gtz);
                const double uy = Gty / konst, uz = Gtz / konst;
                const double cphx = uy * ky + uz * kz;
                const double sphx = sqrt(fmax(0.0, 1.0 - cphx * cphx));
                const double diff = L2 * s2 / (sphx * c2 - cphx * s2);
                const double Kx = ax, Ky = ay + diff * uy, Kz = az + diff * uz;
                const double f = num / (R[0] * Kx + R[3] * Ky + R[6] * Kz);
                const double y2 = f * (R[1] * Kx + R[4] * Ky + R[7] * Kz) + r2d;
                const double z2 = f * (R[2] * Kx + R[5] * Ky + R[8] * Kz) + r3d;
                const double u = dety0 - y2 / pxy, v = detz0 - z2 / pxz;
                if (!(u >= 0.5 && u < ny + 0.5 && v >= 0.5 && v < nz + 0.5)) continue;
                const double iu = floor(u + 0.5), iv = floor(v + 0.5);
                if (iu >= bsy0 && iu <= bsy1 && iv >= bsz0 && iv <= bsz1) continue;
                const int64_t idx = (int64_t)iw * plane + (int64_t)(iu - 1) * nz + (int64_t)(iv - 1);
#pragma omp atomic write
                mask[idx] = 1;
            }
        }
    }
    free(cs);
    free(SUBh);
    return bad ? -2 : 0;
}

/* 1-D squared distance transform of f[0..n) (0 on spot pixels, +Inf elsewhere) into d: the
 * lower envelope of the parabolas (q - p)^2 + f[p]; v and z are scratch of n and n+1 entries. */
static void edt_1d(const double *f, int64_t n, double *d, int64_t *v, double *z) {
    int64_t k = -1;
    for (int64_t q = 0; q < n; ++q) {
        if (isinf(f[q])) continue;
        if (k < 0) {
            k = 0;
            v[0] = q;
            z[0] = -INFINITY;
            z[1] = INFINITY;
            continue;
        }
        double s;
        for (;;) { /* z[0] = -Inf ends the loop at k = 0 at the latest */
            const int64_t p = v[k];
            s = ((f[q] + (double)q * q) - (f[p] + (double)p * p)) / (2.0 * (double)(q - p));
            if (s > z[k]) break;
            --k;
        }
        ++k;
        v[k] = q;
        z[k] = s;
        z[k + 1] = INFINITY;
    }
    if (k < 0) {
        for (int64_t q = 0; q < n; ++q) d[q] = INFINITY;
        return;
    }
    int64_t j = 0;
    for (int64_t q = 0; q < n; ++q) {
        while (z[j + 1] < (double)q) ++j;
        const double t = (double)(q - v[j]);
        d[q] = t * t + f[v[j]];
    }
}

enum { kEdtBlock = 16 };

/* bwdist of each projection: out[iw][y][z] = distance to the nearest mask pixel (float32). */
int host_edt(const uint8_t *mask, int64_t nrot, int64_t ny, int64_t nz, int nthreads, float *out) {
    const int nt = pick_threads(nthreads);
    const int64_t plane = ny * nz, nmax = ny > nz ? ny : nz;
    int fail = 0;
#pragma omp parallel num_threads(nt)
    {
        double *buf = (double *)malloc(sizeof(double) * plane);
        double *ff = (double *)malloc(sizeof(double) * nmax);
        double *z = (double *)malloc(sizeof(double) * (nmax + 1));
        double *blk = (double *)malloc(sizeof(double) * kEdtBlock * ny);
        double *blkd = (double *)malloc(sizeof(double) * kEdtBlock * ny);
        int64_t *v = (int64_t *)malloc(sizeof(int64_t) * nmax);
        if (!buf || !ff || !z || !blk || !blkd || !v) {
#pragma omp atomic write
            fail = 1;
        } else {
#pragma omp for schedule(dynamic, 1)
            for (int64_t iw = 0; iw < nrot; ++iw) {
                const uint8_t *m = mask + iw * plane;
                float *o = out + iw * plane;
                /* pass 1: along detz (contiguous) for every dety row */
                for (int64_t y = 0; y < ny; ++y) {
                    for (int64_t q = 0; q < nz; ++q) ff[q] = m[y * nz + q] ? 0.0 : INFINITY;
                    edt_1d(ff, nz, buf + y * nz, v, z);
                }
                /* pass 2: along dety, kEdtBlock detz columns at a time (row-contiguous gathers) */
                for (int64_t q0 = 0; q0 < nz; q0 += kEdtBlock) {
                    const int64_t nb = nz - q0 < kEdtBlock ? nz - q0 : kEdtBlock;
                    for (int64_t y = 0; y < ny; ++y)
                        for (int64_t b = 0; b < nb; ++b) blk[b * ny + y] = buf[y * nz + q0 + b];
                    for (int64_t b = 0; b < nb; ++b) edt_1d(blk + b * ny, ny, blkd + b * ny, v, z);
                    for (int64_t y = 0; y < ny; ++y)
                        for (int64_t b = 0; b < nb; ++b) o[y * nz + q0 + b] = (float)sqrt(blkd[b * ny + y]);
                }
            }
        }
        free(buf);
        free(ff);
        free(z);
        free(blk);
        free(blkd);
        free(v);
    }
    return fail ? -1 : 0;
}
