/*
 * grc_fit_oracle.c -- TEST INFRASTRUCTURE ONLY (the checker, never the product).
 *
 * FP64 CPU derivatives of the continuous spot landing point, for checking the GPU
 * tangent kernels.  The landing is written in the reference's own formulation
 * (forward_comp.m:17-59: acos of the beam/G angle, atan of the beam tilt, sin of
 * 2*theta and phiy, unit K_out) -- not the algebraic form the GPU uses -- and
 * differentiated by the complex-step method (f'(x) = Im f(x + i h) / h, h = 1e-30),
 * which has no subtractive cancellation, so it is exact to rounding.
 *
 * Parameters: grain g[0..2] = Rodrigues vector (U via quaternion2U.m:3-28 with
 * q0 = 1/sqrt(1+|r|^2), q = r q0), g[3..5] = centre [mm]; geometry e[0..9] = Lsam2sou,
 * Lsam2det, dety00, detz00, tilt_x, tilt_y, tilt_z [deg] (RotDet = Rz*Ry*Rx,
 * get_det_R.m:1-7), P0y, P0z, RotAxisOffset.  Parity status of the landing formula
 * itself: unpinned (see grc_oracle.c).
 */
#include <complex.h>
#include <math.h>

typedef double complex cplx;

static cplx cdot3(const cplx *a, const cplx *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

/* u, v of one reflection; S, B row-major (9), h (3), omega in degrees. */
static void uv_ref(const cplx g[6], const cplx e[10], const double *S, const double *B, const double *h,
                   double omega_deg, double pxy, double pxz, double dety0, double detz0, cplx *u, cplx *v) {
    const double pi = 3.14159265358979323846;
    cplx rr = g[0] * g[0] + g[1] * g[1] + g[2] * g[2];
    cplx q0 = 1.0 / csqrt(1.0 + rr), q1 = g[0] * q0, q2 = g[1] * q0, q3 = g[2] * q0;
    cplx U[9] = {2 * (q0 * q0 + q1 * q1) - 1, 2 * (q1 * q2 - q0 * q3), 2 * (q1 * q3 + q0 * q2),
                 2 * (q1 * q2 + q0 * q3), 2 * (q0 * q0 + q2 * q2) - 1, 2 * (q2 * q3 - q0 * q1),
                 2 * (q1 * q3 - q0 * q2), 2 * (q2 * q3 + q0 * q1), 2 * (q0 * q0 + q3 * q3) - 1};
    cplx Lss = e[0], Lsd = e[1], y00 = e[2], z00 = e[3], P0y = e[7], P0z = e[8], RAO = e[9];
    cplx d2r = pi / 180.0;
    cplx cx = ccos(e[4] * d2r), sx = csin(e[4] * d2r), cy = ccos(e[5] * d2r), sy = csin(e[5] * d2r);
    cplx cz = ccos(e[6] * d2r), sz = csin(e[6] * d2r);
    /* RotDet = Rz*Ry*Rx */
    cplx R[3][3] = {{cz * cy, cz * sy * sx - sz * cx, cz * sy * cx + sz * sx},
                    {sz * cy, sz * sy * sx + cz * cx, sz * sy * cx - cz * sx},
                    {-sy, cy * sx, cy * cx}};
    cplx L = Lss + Lsd;
    /* Gw = S*U*B*h (forward_comp.m:16) */
    double bh[3];
    for (int i = 0; i < 3; ++i) bh[i] = B[3 * i] * h[0] + B[3 * i + 1] * h[1] + B[3 * i + 2] * h[2];
    cplx ubh[3], Gw[3];
    for (int i = 0; i < 3; ++i) ubh[i] = U[3 * i] * bh[0] + U[3 * i + 1] * bh[1] + U[3 * i + 2] * bh[2];
    for (int i = 0; i < 3; ++i) Gw[i] = S[3 * i] * ubh[0] + S[3 * i + 1] * ubh[1] + S[3 * i + 2] * ubh[2];
    cplx pos[3] = {g[3], g[4] - RAO, g[5]}; /* :17 */
    double w = omega_deg * pi / 180.0, co = cos(w), so = sin(w);
    cplx Sp[3];
    for (int i = 0; i < 3; ++i) Sp[i] = S[3 * i] * pos[0] + S[3 * i + 1] * pos[1] + S[3 * i + 2] * pos[2];
    cplx SW[3] = {co * Sp[0] - so * Sp[1], so * Sp[0] + co * Sp[1], Sp[2]}; /* :22 */
    cplx center[3] = {L, (SW[1] - P0y + RAO) * L / (Lss + SW[0]), (SW[2] - P0z) * L / (Lss + SW[0])};
    cplx alpha = catan(csqrt((SW[1] - P0y + RAO) * (SW[1] - P0y + RAO) + (SW[2] - P0z) * (SW[2] - P0z)) /
                       (Lss + SW[0])); /* :25 */
    cplx gp[3] = {Lss + SW[0], SW[1] - P0y + RAO, SW[2] - P0z};
    cplx Gt[3] = {co * Gw[0] - so * Gw[1], so * Gw[0] + co * Gw[1], Gw[2]}; /* :28 */
    cplx Glen = csqrt(cdot3(Gt, Gt));
    cplx ngp = csqrt(cdot3(gp, gp));
    cplx gpu[3] = {gp[0] / ngp, gp[1] / ngp, gp[2] / ngp}, Gtu[3] = {Gt[0] / Glen, Gt[1] / Glen, Gt[2] / Glen};
    cplx beta = cacos(cdot3(gpu, Gtu)); /* :31 */
    cplx theta = beta - pi / 2;
    cplx sintth = csin(2 * theta);
    cplx nv1 = csqrt(Gt[1] * Gt[1] + Gt[2] * Gt[2]);
    cplx ncen = csqrt(cdot3(center, center));
    cplx phix = cacos((Gt[1] / nv1) * (center[1] / ncen) + (Gt[2] / nv1) * (center[2] / ncen)); /* :40 */
    cplx phiy = phix - 2 * theta;
    cplx L2 = (Lsd - SW[0]) / ccos(alpha);
    cplx diffvec = L2 * sintth / csin(phiy);
    cplx konst = nv1;
    cplx y22 = center[1] + diffvec * Gt[1] / konst, z22 = center[2] + diffvec * Gt[2] / konst;
    cplx K[3] = {Lsd - SW[0], y22 - SW[1], z22 - SW[2]};
    cplx nK = csqrt(cdot3(K, K));
    cplx Ku[3] = {K[0] / nK, K[1] / nK, K[2] / nK};
    cplx t = (R[0][0] * (Lsd - SW[0]) + R[1][0] * (y00 - RAO - SW[1]) + R[2][0] * (z00 - SW[2])) /
             (R[0][0] * Ku[0] + R[1][0] * Ku[1] + R[2][0] * Ku[2]); /* :51-52 */
    cplx vv[3] = {t * Ku[0] + SW[0] - Lsd, t * Ku[1] + SW[1] - y00 + RAO, t * Ku[2] + SW[2] - z00};
    cplx y2 = R[0][1] * vv[0] + R[1][1] * vv[1] + R[2][1] * vv[2];
    cplx z2 = R[0][2] * vv[0] + R[1][2] * vv[1] + R[2][2] * vv[2];
    *u = -y2 / pxy + dety0; /* :58 unrounded */
    *v = -z2 / pxz + detz0;
}

/*
 * Landing (u, v) and its Jacobian for one spot.  mode 0: columns over the 6 grain
 * parameters, mode 1: over the 10 geometry parameters.  ju/jv hold 6 or 10 values.
 */
int oracle_fit_uv_jac(int mode, const double *grain6, const double *geo10, const double *S, const double *B,
                      const double *h, double omega_deg, double pxy, double pxz, double dety0, double detz0,
                      double *uv, double *ju, double *jv) {
    const double hstep = 1e-30;
    cplx g[6], e[10], u, v;
    for (int k = 0; k < 6; ++k) g[k] = grain6[k];
    for (int k = 0; k < 10; ++k) e[k] = geo10[k];
    uv_ref(g, e, S, B, h, omega_deg, pxy, pxz, dety0, detz0, &u, &v);
    uv[0] = creal(u);
    uv[1] = creal(v);
    const int K = mode == 0 ? 6 : 10;
    for (int k = 0; k < K; ++k) {
        for (int j = 0; j < 6; ++j) g[j] = grain6[j];
        for (int j = 0; j < 10; ++j) e[j] = geo10[j];
        if (mode == 0)
            g[k] += I * hstep;
        else
            e[k] += I * hstep;
        uv_ref(g, e, S, B, h, omega_deg, pxy, pxz, dety0, detz0, &u, &v);
        ju[k] = cimag(u) / hstep;
        jv[k] = cimag(v) / hstep;
    }
    return 0;
}
