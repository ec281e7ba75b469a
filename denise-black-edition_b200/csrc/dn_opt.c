/*
 * Host parts of the FWI outer loop: the step length from three misfit values
 * (src/calc_opt_step.c, solved here in double) and the bounded model update
 * (src/PSV/calc_mat_change_test_PSV.c, INVMAT1 = 1, the reference's float
 * arithmetic; compiled with -ffp-contract=off).
 */
#include <math.h>
#include <stddef.h>

#include "dn_internal.h"

/* Gaussian elimination with partial pivoting of the 3 x 3 system A x = b */
static int solve3(double A[3][3], double b[3], double x[3])
{
    for (int c = 0; c < 3; c++) {
        int piv = c;
        for (int r = c + 1; r < 3; r++)
            if (fabs(A[r][c]) > fabs(A[piv][c])) piv = r;
        if (A[piv][c] == 0.0) return -1;
        if (piv != c) {
            for (int k = 0; k < 3; k++) {
                double t = A[c][k];
                A[c][k] = A[piv][k];
                A[piv][k] = t;
            }
            double t = b[c];
            b[c] = b[piv];
            b[piv] = t;
        }
        for (int r = c + 1; r < 3; r++) {
            const double f = A[r][c] / A[c][c];
            for (int k = c; k < 3; k++) A[r][k] -= f * A[c][k];
            b[r] -= f * b[c];
        }
    }
    for (int r = 2; r >= 0; r--) {
        double s = b[r];
        for (int k = r + 1; k < 3; k++) s -= A[r][k] * x[k];
        x[r] = s / A[r][r];
    }
    return 0;
}

int dn_calc_opt_step(const double L2t[3], const float epst[3], float *opteps)
{
    if (!L2t || !epst || !opteps) return dn_fail(DN_EINVAL, "dn_calc_opt_step: null argument");
    /* parabola L2(eps) = x0 + x1 eps + x2 eps^2 through the three tests */
    double A[3][3], b[3], x[3];
    for (int i = 0; i < 3; i++) {
        A[i][0] = 1.0;
        A[i][1] = epst[i];
        A[i][2] = (double)epst[i] * (double)epst[i];
        b[i] = L2t[i];
    }
    double eps;
    if (solve3(A, b, x) != 0) {
        eps = epst[0];
    } else {
        eps = -x[1] / (2.0 * x[2]);
        if ((2.0 * x[2]) < 0.0 && L2t[1] > L2t[2]) eps = epst[2];   /* a maximum, still descending */
    }
    if (eps > epst[2]) eps = epst[2];
    if (eps < 0.0 || eps != eps) eps = epst[0];
    *opteps = (float)eps;
    return DN_OK;
}

int dn_mat_update(int nx, int ny, const float *vp, const float *vs, const float *rho, const float *dvp,
                  const float *dvs, const float *drho, float eps_scale, const float lim[6], int iter,
                  const int inv_iter[3], float scalerho, float *vp_out, float *vs_out, float *rho_out,
                  float eps_out[3])
{
    if (!vp || !vs || !rho || !dvp || !dvs || !drho || !lim || !inv_iter || !vp_out || !vs_out || !rho_out ||
        nx < 1 || ny < 1)
        return dn_fail(DN_EINVAL, "dn_mat_update: bad arguments");
    const size_t n = (size_t)nx * ny;
    float pimax = 0.0f, umax = 0.0f, rhomax = 0.0f, gmax = 0.0f, gmax_u = 0.0f, gmax_rho = 0.0f;
    for (size_t k = 0; k < n; k++) {
        if (vp[k] > pimax) pimax = vp[k];
        if (vs[k] > umax) umax = vs[k];
        if (rho[k] > rhomax) rhomax = rho[k];
        if (fabsf(dvp[k]) > gmax) gmax = fabsf(dvp[k]);
        if (fabsf(dvs[k]) > gmax_u) gmax_u = fabsf(dvs[k]);
        if (fabsf(drho[k]) > gmax_rho) gmax_rho = fabsf(drho[k]);
    }
    float eps = eps_scale * (pimax / gmax);
    float eps_u = eps_scale * (umax / gmax_u);
    float eps_rho = eps_scale * (rhomax / gmax_rho) * scalerho;
    if (iter < inv_iter[0]) eps = 0.0f;
    if (iter < inv_iter[1]) eps_u = 0.0f;
    if (iter < inv_iter[2]) eps_rho = 0.0f;
    for (size_t k = 0; k < n; k++) {
        float p = vp[k] - eps * dvp[k];
        float u = vs[k] - eps_u * dvs[k];
        float r = rho[k] - eps_rho * drho[k];
        if (p < lim[0] || p > lim[1]) p = vp[k];
        if ((u < lim[2] && u > 1e-6) || u > lim[3]) u = vs[k];
        if (r < lim[4] || r > lim[5]) r = rho[k];
        if (p < 0.0f) p = vp[k];
        if (u < 0.0f) u = vs[k];
        if (r < 0.0f) r = rho[k];
        vp_out[k] = p;
        vs_out[k] = u;
        rho_out[k] = r;
    }
    if (eps_out) {
        eps_out[0] = eps;
        eps_out[1] = eps_u;
        eps_out[2] = eps_rho;
    }
    return DN_OK;
}
