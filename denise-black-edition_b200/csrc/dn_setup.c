/*
 * Host set-up numerics of the P-SV path: FD coefficients, CPML profiles,
 * staggered material averages, viscoelastic coefficients and source wavelets.
 *
 * These run once per model / shot on the host and must be bit-identical to
 * the reference, so every expression keeps the reference's C evaluation
 * order and its float -> double promotions (a float operand meeting a double
 * literal is widened, the sum/product is rounded once in double and the
 * assignment rounds to float).  The file is compiled with
 * -ffp-contract=off -fno-fast-math so the compiler may not fuse or reorder.
 * glibc's exp/log/pow are the same functions the reference calls.
 */
#include "denise_b200.h"
#include "dn_internal.h"

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define DN_PI (3.141592653589793)

/* ------------------------------------------------------------------------
 * Finite-difference coefficients.
 * Staggered-grid Taylor coefficients (E = 0) and Holberg's group-velocity
 * optimised coefficients for relative errors E = 0.1 %, 0.5 %, 1 %, 3 %, for
 * half-orders 1..6.  Column 0 is the minimum number of grid points per
 * shortest wavelength.  Same published values as src/holbergcoeff.c:25-67;
 * each entry is rounded from its double value to float exactly as the
 * reference's float initialiser does.
 * ------------------------------------------------------------------------ */
static const double dn_fd_table[5][6][7] = {
    /* E = 0: Taylor */
    {{23.0, 1.0, 0, 0, 0, 0, 0},
     {8.0, 9.0 / 8.0, -1.0 / 24.0, 0, 0, 0, 0},
     {6.0, 75.0 / 64.0, -25.0 / 384.0, 3.0 / 640.0, 0, 0, 0},
     {5.0, 1225.0 / 1024.0, -245.0 / 3072.0, 49.0 / 5120.0, -5.0 / 7168.0, 0, 0},
     {5.0, 19845.0 / 16384.0, -735.0 / 8192.0, 567.0 / 40960.0, -405.0 / 229376.0, 35.0 / 294912.0, 0},
     {4.0, 160083.0 / 131072.0, -12705.0 / 131072.0, 22869.0 / 1310720.0, -5445.0 / 1835008.0,
      847.0 / 2359296.0, -63.0 / 2883584.0}},
    /* E = 0.1 % */
    {{49.7, 1.0010, 0, 0, 0, 0, 0},
     {8.32, 1.1382, -0.046414, 0, 0, 0, 0},
     {4.77, 1.1965, -0.078804, 0.0081781, 0, 0, 0},
     {3.69, 1.2257, -0.099537, 0.018063, -0.0026274, 0, 0},
     {3.19, 1.2415, -0.11231, 0.026191, -0.0064682, 0.001191, 0},
     {2.91, 1.2508, -0.12034, 0.032131, -0.010142, 0.0029857, -0.00066667}},
    /* E = 0.5 % */
    {{22.2, 1.0050, 0, 0, 0, 0, 0},
     {5.65, 1.1534, -0.052806, 0, 0, 0, 0},
     {3.74, 1.2111, -0.088313, 0.011768, 0, 0, 0},
     {3.11, 1.2367, -0.10815, 0.023113, -0.0046905, 0, 0},
     {2.80, 1.2496, -0.11921, 0.031130, -0.0093272, 0.0025161, 0},
     {2.62, 1.2568, -0.12573, 0.036423, -0.013132, 0.0047484, -0.0015979}},
    /* E = 1 % */
    {{15.8, 1.0100, 0, 0, 0, 0, 0},
     {4.80, 1.1640, -0.057991, 0, 0, 0, 0},
     {3.39, 1.2192, -0.094070, 0.014608, 0, 0, 0},
     {2.90, 1.2422, -0.11269, 0.026140, -0.0064054, 0, 0},
     {2.65, 1.2534, -0.12257, 0.033755, -0.011081, 0.0036784, 0},
     {2.51, 1.2596, -0.12825, 0.038550, -0.014763, 0.0058619, -0.0024538}},
    /* E = 3 % */
    {{9.16, 1.0300, 0, 0, 0, 0, 0},
     {3.47, 1.1876, -0.072518, 0, 0, 0, 0},
     {2.91, 1.2341, -0.10569, 0.022589, 0, 0, 0},
     {2.61, 1.2516, -0.12085, 0.032236, -0.011459, 0, 0},
     {2.45, 1.2596, -0.12829, 0.038533, -0.014681, 0.0072580, 0},
     {2.36, 1.2640, -0.13239, 0.042217, -0.017803, 0.0081959, -0.0051848}},
};

int dn_holbergcoeff(int fdorder, int maxrelerror, float hc[7])
{
    if (fdorder < 2 || fdorder > 12 || (fdorder % 2) != 0)
        return dn_fail(DN_EINVAL, "Error in selection of FD coefficients: wrong FDORDER (%d)", fdorder);
    if (maxrelerror < 0 || maxrelerror > 4)
        return dn_fail(DN_EINVAL, "Error in selection of FD coefficients: wrong choice of maximum relative error (%d)",
                       maxrelerror);
    int row = fdorder / 2 - 1;
    for (int k = 0; k <= 6; k++) hc[k] = (float)dn_fd_table[maxrelerror][row][k];
    return DN_OK;
}

/* ------------------------------------------------------------------------
 * CPML damping profiles, src/PML_pro.c:65-407 (single subdomain: NXG = NX).
 * ------------------------------------------------------------------------ */
static void pml_edge(float *d, float *K, float *alpha, float *a, float *b, float d0, float abscissa,
                     float thickness, float npower, float k_max, float alpha_max, int clamp_alpha, float DT)
{
    if (abscissa >= 0.0) {
        float an = abscissa / thickness;
        *d = d0 * pow(an, npower);                            /* float * double -> float */
        *K = 1.0 + (k_max - 1.0) * pow(an, npower);
        *alpha = alpha_max * (1.0 - an);
    }
    if (clamp_alpha && *alpha < 0.0) *alpha = 0.0;
    (void)a; (void)b; (void)DT;
}

static void pml_ab(float d, float K, float alpha, float *a, float *b, float DT)
{
    float arg = -(d / K + alpha) * DT;                         /* all float */
    *b = exp(arg);
    /* integer abs() on the float, as PML_pro.c:153: a is set only where |(int)d| >= 1 */
    if (abs((int)d) > 1.0e-6) *a = d * (*b - 1.0) / (K * (d + K * alpha));
}

int dn_pml_profiles(const dn_params *p, dn_pml *o)
{
    if (!p || !o) return dn_fail(DN_EINVAL, "dn_pml_profiles: null argument");
    const int FW = p->fw;
    if (FW <= 0) return DN_OK;
    const float DH = p->dh, DT = p->dt, DAMPING = p->damping, FPML = p->fpml;
    const float npower = p->npower, k_max_PML = p->k_max_pml;
    const int NXG = p->nx, NYG = p->ny;
    float *vecs[20] = {o->d_x, o->K_x, o->alpha_prime_x, o->a_x, o->b_x,
                       o->d_x_half, o->K_x_half, o->alpha_prime_x_half, o->a_x_half, o->b_x_half,
                       o->d_y, o->K_y, o->alpha_prime_y, o->a_y, o->b_y,
                       o->d_y_half, o->K_y_half, o->alpha_prime_y_half, o->a_y_half, o->b_y_half};
    for (int k = 0; k < 20; k++) {
        if (!vecs[k]) return dn_fail(DN_EINVAL, "dn_pml_profiles: vector %d is NULL", k);
        memset(vecs[k], 0, sizeof(float) * 2 * (size_t)FW);   /* vector() zero-initialises */
    }
    /* 1-based views */
    float *d_x = o->d_x - 1, *K_x = o->K_x - 1, *al_x = o->alpha_prime_x - 1, *a_x = o->a_x - 1, *b_x = o->b_x - 1;
    float *d_xh = o->d_x_half - 1, *K_xh = o->K_x_half - 1, *al_xh = o->alpha_prime_x_half - 1;
    float *a_xh = o->a_x_half - 1, *b_xh = o->b_x_half - 1;
    float *d_y = o->d_y - 1, *K_y = o->K_y - 1, *al_y = o->alpha_prime_y - 1, *a_y = o->a_y - 1, *b_y = o->b_y - 1;
    float *d_yh = o->d_y_half - 1, *K_yh = o->K_y_half - 1, *al_yh = o->alpha_prime_y_half - 1;
    float *a_yh = o->a_y_half - 1, *b_yh = o->b_y_half - 1;

    const float alpha_max_PML = 2.0 * DN_PI * (FPML / 2.0);
    float thickness_PML_x = FW * DH;
    float thickness_PML_y = FW * DH;
    float Rcoef = 0.001;
    float d0_x = -(npower + 1) * DAMPING * log(Rcoef) / (2.0 * thickness_PML_x);
    float d0_y = -(npower + 1) * DAMPING * log(Rcoef) / (2.0 * thickness_PML_y);

    /* x: left frame h = i, right frame h = i - NXG + 2 FW */
    float xoriginleft = thickness_PML_x;
    float xoriginright = (NXG - 1) * DH - thickness_PML_x;
    for (int i = 1; i <= FW; i++) {
        K_x[i] = 1.0;
        K_xh[i] = 1.0;
        float xval = DH * (i - 1);
        float ab = xoriginleft - xval;
        pml_edge(&d_x[i], &K_x[i], &al_x[i], 0, 0, d0_x, ab, thickness_PML_x, npower, k_max_PML, alpha_max_PML, 0, DT);
        ab = xoriginleft - (xval + DH / 2.0);
        pml_edge(&d_xh[i], &K_xh[i], &al_xh[i], 0, 0, d0_x, ab, thickness_PML_x, npower, k_max_PML, alpha_max_PML, 0,
                 DT);
        if (al_x[i] < 0.0) al_x[i] = 0.0;
        if (al_xh[i] < 0.0) al_xh[i] = 0.0;
        pml_ab(d_x[i], K_x[i], al_x[i], &a_x[i], &b_x[i], DT);
        pml_ab(d_xh[i], K_xh[i], al_xh[i], &a_xh[i], &b_xh[i], DT);
    }
    for (int i = NXG - FW + 1; i <= NXG; i++) {
        int h = i - NXG + 2 * FW;
        K_x[h] = 1.0;
        K_xh[h] = 1.0;
        float xval = DH * (i - 1);
        float ab = xval - xoriginright;
        pml_edge(&d_x[h], &K_x[h], &al_x[h], 0, 0, d0_x, ab, thickness_PML_x, npower, k_max_PML, alpha_max_PML, 0, DT);
        ab = xval + DH / 2.0 - xoriginright;
        pml_edge(&d_xh[h], &K_xh[h], &al_xh[h], 0, 0, d0_x, ab, thickness_PML_x, npower, k_max_PML, alpha_max_PML, 0,
                 DT);
        if (al_x[h] < 0.0) al_x[h] = 0.0;
        if (al_xh[h] < 0.0) al_xh[h] = 0.0;
        pml_ab(d_x[h], K_x[h], al_x[h], &a_x[h], &b_x[h], DT);
        pml_ab(d_xh[h], K_xh[h], al_xh[h], &a_xh[h], &b_xh[h], DT);
    }
    /* y: top frame h = j (no alpha clamp in the reference), bottom h = j - NYG + 2 FW */
    float yoriginbottom = thickness_PML_y;
    float yorigintop = (NYG - 1) * DH - thickness_PML_y;
    for (int i = 1; i <= FW; i++) {
        K_y[i] = 1.0;
        K_yh[i] = 1.0;
        float yval = DH * (i - 1);
        float ab = yoriginbottom - yval;
        pml_edge(&d_y[i], &K_y[i], &al_y[i], 0, 0, d0_y, ab, thickness_PML_y, npower, k_max_PML, alpha_max_PML, 0, DT);
        ab = yoriginbottom - (yval + DH / 2.0);
        pml_edge(&d_yh[i], &K_yh[i], &al_yh[i], 0, 0, d0_y, ab, thickness_PML_y, npower, k_max_PML, alpha_max_PML, 0,
                 DT);
        pml_ab(d_y[i], K_y[i], al_y[i], &a_y[i], &b_y[i], DT);
        pml_ab(d_yh[i], K_yh[i], al_yh[i], &a_yh[i], &b_yh[i], DT);
    }
    for (int i = NYG - FW + 1; i <= NYG; i++) {
        int h = i - NYG + 2 * FW;
        K_y[h] = 1.0;
        K_yh[h] = 1.0;
        float yval = DH * (i - 1);
        float ab = yval - yorigintop;
        pml_edge(&d_y[h], &K_y[h], &al_y[h], 0, 0, d0_y, ab, thickness_PML_y, npower, k_max_PML, alpha_max_PML, 0, DT);
        ab = yval + DH / 2.0 - yorigintop;
        /* the reference scales this half-grid profile with d0_x (PML_pro.c:281); equal to d0_y here */
        pml_edge(&d_yh[h], &K_yh[h], &al_yh[h], 0, 0, d0_x, ab, thickness_PML_y, npower, k_max_PML, alpha_max_PML, 0,
                 DT);
        pml_ab(d_y[h], K_y[h], al_y[h], &a_y[h], &b_y[h], DT);
        pml_ab(d_yh[h], K_yh[h], al_yh[h], &a_yh[h], &b_yh[h], DT);
    }
    return DN_OK;
}

/* ------------------------------------------------------------------------
 * CFL limit, src/checkfd_ssg_elastic.c:89,126 (hc[1..6] all entries used).
 * ------------------------------------------------------------------------ */
int dn_cfl_check(const dn_params *p, float vp_max, double *dtstab)
{
    float hc[7];
    int st = dn_holbergcoeff(p->fdorder, p->maxrelerror, hc);
    if (st) return st;
    float gamma = fabs(hc[1]) + fabs(hc[2]) + fabs(hc[3]) + fabs(hc[4]) + fabs(hc[5]) + fabs(hc[6]);
    float ds = p->dh / (sqrt(2) * gamma * vp_max);
    if (dtstab) *dtstab = ds;
    if (p->dt > ds)
        return dn_fail(DN_EINVAL, "The simulation will get unstable, choose smaller DT (DT=%g > dtstab=%g)",
                       (double)p->dt, (double)ds);
    return DN_OK;
}

/* ------------------------------------------------------------------------
 * Material halo: the reference reads the model into [1..NY][1..NX] and
 * matcopy_*_PSV fills rows 0 / NY+1 and then columns 0 / NX+1 from the
 * opposite edge (on one rank every neighbour is the rank itself).
 * ------------------------------------------------------------------------ */
typedef struct {
    int nx, ny;
    float *a; /* (ny+2) x (nx+2), index (j, i) for j = 0..ny+1, i = 0..nx+1 */
} halo_grid;

static float *hg_at(halo_grid *g, int j, int i) { return &g->a[(size_t)j * (g->nx + 2) + i]; }

static int hg_from_file(halo_grid *g, int nx, int ny, const float *file)
{
    g->nx = nx;
    g->ny = ny;
    g->a = (float *)calloc((size_t)(nx + 2) * (ny + 2), sizeof(float));
    if (!g->a) return DN_ENOMEM;
    for (int i = 1; i <= nx; i++)
        for (int j = 1; j <= ny; j++) *hg_at(g, j, i) = file[(size_t)(i - 1) * ny + (j - 1)];
    /* matcopy: rows first (columns 0..NX+1, still zero at the corners) */
    for (int i = 0; i <= nx + 1; i++) {
        float top = *hg_at(g, 1, i), bot = *hg_at(g, ny, i);
        *hg_at(g, ny + 1, i) = top;
        *hg_at(g, 0, i) = bot;
    }
    /* then columns, rows 0..NY+1 */
    for (int j = 0; j <= ny + 1; j++) {
        float left = *hg_at(g, j, 1), right = *hg_at(g, j, nx);
        *hg_at(g, j, nx + 1) = left;
        *hg_at(g, j, 0) = right;
    }
    return DN_OK;
}

int dn_average_materials(const dn_params *p, const float *vp, const float *vs, const float *rho, float *uipjp,
                         float *rip, float *rjp)
{
    if (!p || !vp || !vs || !rho) return dn_fail(DN_EINVAL, "dn_average_materials: null argument");
    if (p->invmat1 != 1) return dn_fail(DN_ENOTSUP, "dn_average_materials: only INVMAT1=1 (vp, vs, rho) is supported");
    const int nx = p->nx, ny = p->ny;
    halo_grid R = {0}, U = {0};
    int st = hg_from_file(&R, nx, ny, rho);
    if (!st) st = hg_from_file(&U, nx, ny, vs);
    if (st) {
        free(R.a);
        free(U.a);
        return dn_fail(DN_ENOMEM, "dn_average_materials: out of host memory");
    }
    (void)vp;
    for (int j = 1; j <= ny; j++) {
        for (int i = 1; i <= nx; i++) {
            size_t o = (size_t)(i - 1) * ny + (j - 1);
            if (uipjp) {
                /* av_mue.c:29-44 (INVMAT1 == 1) */
                float u1 = *hg_at(&R, j, i) * *hg_at(&U, j, i) * *hg_at(&U, j, i);
                float u2 = *hg_at(&R, j, i + 1) * *hg_at(&U, j, i + 1) * *hg_at(&U, j, i + 1);
                float u3 = *hg_at(&R, j + 1, i) * *hg_at(&U, j + 1, i) * *hg_at(&U, j + 1, i);
                float u4 = *hg_at(&R, j + 1, i + 1) * *hg_at(&U, j + 1, i + 1) * *hg_at(&U, j + 1, i + 1);
                float v = 4.0 / ((1.0 / u1) + (1.0 / u2) + (1.0 / u3) + (1.0 / u4));
                if ((u1 == 0.0) || (u2 == 0.0) || (u3 == 0.0) || (u4 == 0.0)) v = 0.0;
                uipjp[o] = v;
            }
            /* av_rho.c:13-22 */
            float r00 = *hg_at(&R, j, i), r10 = *hg_at(&R, j + 1, i), r01 = *hg_at(&R, j, i + 1);
            float vj = 1.0 / (0.5 * (r00 + r10));
            float vi = 1.0 / (0.5 * (r00 + r01));
            if ((r00 < 1e-4) && (r10 < 1e-4)) vj = 0.0;
            if ((r00 < 1e-4) && (r01 < 1e-4)) vi = 0.0;
            if (rjp) rjp[o] = vj;
            if (rip) rip[o] = vi;
        }
    }
    free(R.a);
    free(U.a);
    return DN_OK;
}

/* ------------------------------------------------------------------------
 * Viscoelastic coefficients.
 * ------------------------------------------------------------------------ */
int dn_visc_eta(const dn_params *p, float *eta, float *pts)
{
    /* readmod_visc_PSV.c:31-35 */
    for (int l = 0; l < p->L; l++) {
        float t = 1.0 / (2.0 * DN_PI * p->fl[l]);
        if (pts) pts[l] = t;
        eta[l] = p->dt / t;
    }
    return DN_OK;
}

float dn_visc_sum(const dn_params *p, float ws)
{
    /* prepare_update_s_visc_PSV.c:37-41 / surface_visc_PML_PSV.c:45-49: float accumulation
       of a double quotient */
    float sumu = 0.0;
    for (int l = 0; l < p->L; l++) {
        float pt = 1.0 / (2.0 * DN_PI * p->fl[l]);
        sumu = sumu + ((ws * ws * pt * pt) / (1.0 + ws * ws * pt * pt));
    }
    return sumu;
}

float dn_visc_tau_from_q(float q)
{
    /* readmod_visc_PSV.c:119-120: taus = 2/Qs, taup = 2/Qp */
    return 2.0 / q;
}

int dn_prepare_visc(const dn_params *p, const float *vp, const float *vs, const float *rho, const float *qp,
                    const float *qs, float *fipjp, float *f, float *g, float *dip, float *d, float *e, float *bip,
                    float *bjm, float *cip, float *cjm, float *eta_out)
{
    if (!p || p->L < 1 || p->L > DN_MAX_L) return dn_fail(DN_EINVAL, "dn_prepare_visc: L must be in 1..%d", DN_MAX_L);
    if (p->invmat1 != 1) return dn_fail(DN_ENOTSUP, "dn_prepare_visc: only INVMAT1=1 is supported");
    if (p->honor_q && (!qp || !qs)) return dn_fail(DN_EINVAL, "dn_prepare_visc: honor_q needs qp and qs");
    const int nx = p->nx, ny = p->ny, L = p->L;
    const size_t n = (size_t)nx * ny;
    float eta[DN_MAX_L];
    dn_visc_eta(p, eta, NULL);
    float *tausf = (float *)malloc(n * sizeof(float));
    float *taupf = (float *)malloc(n * sizeof(float));
    float *uipjp = (float *)malloc(n * sizeof(float));
    if (!tausf || !taupf || !uipjp) {
        free(tausf);
        free(taupf);
        free(uipjp);
        return dn_fail(DN_ENOMEM, "dn_prepare_visc: out of host memory");
    }
    for (size_t k = 0; k < n; k++) {
        float qpv = p->honor_q ? qp[k] : 30.0f;   /* readmod_visc_PSV.c:106-107 forces Q = 30 */
        float qsv = p->honor_q ? qs[k] : 30.0f;
        tausf[k] = dn_visc_tau_from_q(qsv);
        taupf[k] = dn_visc_tau_from_q(qpv);
    }
    int st = dn_average_materials(p, vp, vs, rho, uipjp, NULL, NULL);
    halo_grid T = {0};
    if (!st) st = hg_from_file(&T, nx, ny, tausf);
    if (st) {
        free(tausf);
        free(taupf);
        free(uipjp);
        free(T.a);
        return st ? st : DN_ENOMEM;
    }
    /* prepare_update_s_visc_PSV.c:28-41 */
    float ws = 2.0 * DN_PI * p->fl[0];
    float sumu = dn_visc_sum(p, ws);
    float sumpi = sumu;
    for (int l = 0; l < L; l++) {
        if (bip) bip[l] = 1.0 / (1.0 + (eta[l] * 0.5));
        if (bjm) bjm[l] = 1.0 / (1.0 + (eta[l] * 0.5));
        if (cip) cip[l] = 1.0 - (eta[l] * 0.5);
        if (cjm) cjm[l] = 1.0 - (eta[l] * 0.5);
        if (eta_out) eta_out[l] = eta[l];
    }
    const float DT = p->dt;
    for (int j = 1; j <= ny; j++) {
        for (int i = 1; i <= nx; i++) {
            size_t o = (size_t)(i - 1) * ny + (j - 1);
            /* av_tau.c:13 */
            float tsij = 0.25 * (*hg_at(&T, j, i) + *hg_at(&T, j, i + 1) + *hg_at(&T, j + 1, i) + *hg_at(&T, j + 1, i + 1));
            float pu = vs[o], ppi = vp[o], prho = rho[o];
            float mu = (pu * pu * prho) / (1.0 + sumu * tausf[o]);
            float pi = (ppi * ppi * prho) / (1.0 + sumpi * taupf[o]);
            float muipjp = uipjp[o] / (1.0 + sumu * tsij);
            if (fipjp) fipjp[o] = muipjp * DT * (1.0 + L * tsij);
            if (f) f[o] = mu * DT * (1.0 + L * tausf[o]);
            if (g) g[o] = pi * DT * (1.0 + L * taupf[o]);
            for (int l = 0; l < L; l++) {
                if (dip) dip[(size_t)l * n + o] = muipjp * eta[l] * tsij;
                if (d) d[(size_t)l * n + o] = mu * eta[l] * tausf[o];
                if (e) e[(size_t)l * n + o] = pi * eta[l] * taupf[o];
            }
        }
    }
    free(tausf);
    free(taupf);
    free(uipjp);
    free(T.a);
    return DN_OK;
}

/* Per-cell "relaxed modulus" factors the device regenerates the visco
 * coefficients from (fipjp, f, g, dip, d, e) without storing the 3L arrays:
 *   muipjp, tausipjp, mu, taus, pi, taup  (prepare_update_s_visc_PSV.c:46-60).
 * Outputs in file order. */
float dn_visc_sumu(const dn_params *p)
{
    float ws = 2.0 * DN_PI * p->fl[0];
    return dn_visc_sum(p, ws);
}

int dn_visc_cell_factors(const dn_params *p, const float *vp, const float *vs, const float *rho, const float *qp,
                         const float *qs, float *muipjp_o, float *tausipjp_o, float *mu_o, float *taus_o, float *pi_o,
                         float *taup_o)
{
    const int nx = p->nx, ny = p->ny;
    const size_t n = (size_t)nx * ny;
    float *uipjp = (float *)malloc(n * sizeof(float));
    float *tausf = (float *)malloc(n * sizeof(float));
    if (!uipjp || !tausf) {
        free(uipjp);
        free(tausf);
        return dn_fail(DN_ENOMEM, "dn_visc_cell_factors: out of host memory");
    }
    for (size_t k = 0; k < n; k++) tausf[k] = dn_visc_tau_from_q(p->honor_q ? qs[k] : 30.0f);
    int st = dn_average_materials(p, vp, vs, rho, uipjp, NULL, NULL);
    halo_grid T = {0};
    if (!st) st = hg_from_file(&T, nx, ny, tausf);
    if (st) {
        free(uipjp);
        free(tausf);
        free(T.a);
        return st;
    }
    float sumu = dn_visc_sumu(p);
    for (int i = 1; i <= nx; i++) {       /* cells are independent: file order, contiguous in o */
        for (int j = 1; j <= ny; j++) {
            size_t o = (size_t)(i - 1) * ny + (j - 1);
            float tsij = 0.25 * (*hg_at(&T, j, i) + *hg_at(&T, j, i + 1) + *hg_at(&T, j + 1, i) + *hg_at(&T, j + 1, i + 1));
            float tp = dn_visc_tau_from_q(p->honor_q ? qp[o] : 30.0f);
            float pu = vs[o], ppi = vp[o], prho = rho[o];
            muipjp_o[o] = uipjp[o] / (1.0 + sumu * tsij);
            tausipjp_o[o] = tsij;
            mu_o[o] = (pu * pu * prho) / (1.0 + sumu * tausf[o]);
            taus_o[o] = tausf[o];
            pi_o[o] = (ppi * ppi * prho) / (1.0 + sumu * tp);
            taup_o[o] = tp;
        }
    }
    free(uipjp);
    free(tausf);
    free(T.a);
    return DN_OK;
}

/* ------------------------------------------------------------------------
 * Source wavelets, src/wavelet.c:33-106: QUELLART 1 Ricker, 2 fuchs-mueller,
 * 3 samples from a file, 4 sin^3, 5 first derivative of a Gaussian, 6 spike
 * (band-limited afterwards by the caller, FD_PSV.c:324-331), 7 Klauder
 * (chirp from FC_SPIKE_1 to FC_SPIKE_2 over TS), then the N_ORDER
 * integration of :97-106.  Float and double operations in the order and
 * precision of the reference's expressions.
 * ------------------------------------------------------------------------ */
int dn_wavelet_ex(int quellart, int nt, float DT, float tshift, float fc, float a, int n_order, float fc_spike_1,
                  float fc_spike_2, float ts_chirp, const float *file_signal, int file_ns, float *out)
{
    if (!out || nt < 1) return dn_fail(DN_EINVAL, "dn_wavelet: bad arguments");
    if (quellart == 3 && (!file_signal || file_ns < nt))
        return dn_fail(DN_EINVAL, "QUELLART 3: the wavelet file holds %d samples, NT = %d", file_signal ? file_ns : 0, nt);
    float k1 = 0.0f, f0 = 0.0f;
    if (quellart == 7) {
        k1 = (fc_spike_2 - fc_spike_1) / ts_chirp;   /* rate of change of the frequency */
        f0 = (fc_spike_2 + fc_spike_1) / 2.0;        /* mid frequency */
    }
    for (int k = 1; k <= nt; k++) {
        float t = (float)k * DT;
        float ts = 1.0 / fc;
        float ag = DN_PI * DN_PI * fc * fc;
        float amp = 0.0, tau, t1;
        switch (quellart) {
        case 1:
            tau = DN_PI * (t - 1.5 * ts - tshift) / (1.5 * ts);
            amp = (((1.0 - 4.0 * tau * tau) * exp(-2.0 * tau * tau)));
            break;
        case 2:
            if ((t < tshift) || (t > (tshift + ts))) amp = 0.0;
            else amp = ((sin(2.0 * DN_PI * (t - tshift) * fc) - 0.5 * sin(4.0 * DN_PI * (t - tshift) * fc)));
            break;
        case 3:
            amp = file_signal[k - 1];
            break;
        case 4:
            if ((t < tshift) || (t > (tshift + ts))) amp = 0.0;
            else amp = pow(sin(DN_PI * (t + tshift) / ts), 3.0);
            break;
        case 5:
            ts = 1.2 / fc;
            ag = DN_PI * DN_PI * fc * fc;
            amp = -2.0 * ag * (t - ts) * exp(-ag * (t - ts) * (t - ts));
            break;
        case 6:
            amp = 0.0;
            if (k == 1 + (int)floor(tshift / DT + 0.5)) amp = 1.0;
            break;
        case 7:
            ts = 1.5 / fc_spike_1;
            t1 = t - ts - tshift;
            amp = creal(cexp(0.0 + 2.0 * DN_PI * f0 * t1 * I) * sin(DN_PI * k1 * t1 * (ts_chirp - t1)) /
                        (DN_PI * k1 * t1));
            break;
        default:
            return dn_fail(DN_ENOTSUP, "Which source-wavelet ? (QUELLART=%d)", quellart);
        }
        out[k - 1] = amp * a;
    }
    for (int r = 1; r <= n_order; r++) {
        out[0] = out[0] * DT;
        for (int k = 2; k <= nt; k++) out[k - 1] = out[k - 2] + out[k - 1] * DT;
    }
    return DN_OK;
}

int dn_wavelet(int quellart, int nt, float DT, float tshift, float fc, float a, int n_order, float *out)
{
    if (quellart == 3 || quellart == 7)
        return dn_fail(DN_EINVAL, "dn_wavelet: QUELLART %d needs dn_wavelet_ex (file samples / chirp band)", quellart);
    return dn_wavelet_ex(quellart, nt, DT, tshift, fc, a, n_order, 0.0f, 0.0f, 0.0f, NULL, 0, out);
}
