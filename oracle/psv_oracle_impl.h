/*
 * ORACLE / TEST INFRASTRUCTURE - body of the CPU restatement, included twice
 * by psv_oracle.c with REAL = float (suffix _f) and REAL = double (_d).
 * The per-cell loops of the updates, the snapshot store and the correlation
 * run in parallel over rows (OpenMP): every iteration writes only its own
 * cells, so the results do not depend on the thread count.
 * Variables the reference declares `float` are REAL here; every double
 * literal and double intermediate of the reference is kept, so the _f build
 * reproduces the reference's rounding and the _d build is an FP64 scheme.
 */

#define CTX OR_CAT(or_ctx, SFX)
#define FN(name) OR_CAT(name, SFX)
#define H 8
#define AT(a, j, i) (a)[(size_t)((j) + H) * c->pitch + (size_t)((i) + H)]
#define XF(a, j, h) (a)[(size_t)(j) * (2 * c->fw + 1) + (h)]   /* x frame psi[j][h], 1-based */
#define ZF(a, h, i) (a)[(size_t)(h) * (c->nx + 1) + (i)]       /* z frame psi[h][i], 1-based */
#define FO(i, j) ((size_t)((i) - 1) * c->ny + ((j) - 1))        /* file-order index */

struct CTX {
    int nx, ny, nt, R, maxrel, free_surf, fw, L, quelltypb, dtinv, seismo, eprecond, honor_q;
    REAL dh, dt, damping, fpml, npower, kmax, ts, fl[6];
    REAL hc[7];
    int pitch, rows;
    size_t plane;
    REAL *vx, *vy, *sxx, *syy, *sxy, *vxp1, *vyp1, *r, *p, *q;
    REAL *rho, *pi, *u, *rip, *rjp, *uipjp, *taus, *taup, *tausipjp;
    REAL *fipjp, *f, *g, *dip, *d, *e;
    REAL eta[6], bip[6], bjm[6], cip[6], cjm[6];
    REAL *K_x, *a_x, *b_x, *K_xh, *a_xh, *b_xh, *K_y, *a_y, *b_y, *K_yh, *a_yh, *b_yh;
    REAL *d_x, *al_x, *d_xh, *al_xh, *d_y, *al_y, *d_yh, *al_yh;
    REAL *psi_sxx_x, *psi_sxy_x, *psi_vxx, *psi_vyx, *psi_vxxs, *psi_syy_y, *psi_sxy_y, *psi_vyy, *psi_vxy;
    int nsrc, ntr, quelltyp;
    int *src_i, *src_j, *src_type, *rec_i, *rec_j;
    REAL *src_azi;
    REAL *signals;          /* [nsrc][nt+1], 1-based time */
    REAL *sec;              /* [5][ntr][nt+1] */
    REAL *res[3];           /* [ntr][nt+1] */
    int nsnap;
    REAL *snap;             /* [nsnap][5][nx*ny] file order */
    REAL *wc, *wcu, *wcr, *Ws, *Wr;   /* file order */
    REAL *gvp, *gvs, *grho;
};

static void *FN(or_zalloc)(size_t n, size_t s)
{
    void *p = calloc(n ? n : 1, s);
    if (!p) {
        fprintf(stderr, "oracle: out of memory\n");
        abort();
    }
    return p;
}

/* holbergcoeff.c:25-86 */
static void FN(or_hc)(CTX *c)
{
    static const double tab[5][6][7] = {
        {{23.0, 1.0, 0, 0, 0, 0, 0}, {8.0, 9.0 / 8.0, -1.0 / 24.0, 0, 0, 0, 0},
         {6.0, 75.0 / 64.0, -25.0 / 384.0, 3.0 / 640.0, 0, 0, 0},
         {5.0, 1225.0 / 1024.0, -245.0 / 3072.0, 49.0 / 5120.0, -5.0 / 7168.0, 0, 0},
         {5.0, 19845.0 / 16384.0, -735.0 / 8192.0, 567.0 / 40960.0, -405.0 / 229376.0, 35.0 / 294912.0, 0},
         {4.0, 160083.0 / 131072.0, -12705.0 / 131072.0, 22869.0 / 1310720.0, -5445.0 / 1835008.0, 847.0 / 2359296.0,
          -63.0 / 2883584.0}},
        {{49.7, 1.0010, 0, 0, 0, 0, 0}, {8.32, 1.1382, -0.046414, 0, 0, 0, 0},
         {4.77, 1.1965, -0.078804, 0.0081781, 0, 0, 0}, {3.69, 1.2257, -0.099537, 0.018063, -0.0026274, 0, 0},
         {3.19, 1.2415, -0.11231, 0.026191, -0.0064682, 0.001191, 0},
         {2.91, 1.2508, -0.12034, 0.032131, -0.010142, 0.0029857, -0.00066667}},
        {{22.2, 1.0050, 0, 0, 0, 0, 0}, {5.65, 1.1534, -0.052806, 0, 0, 0, 0},
         {3.74, 1.2111, -0.088313, 0.011768, 0, 0, 0}, {3.11, 1.2367, -0.10815, 0.023113, -0.0046905, 0, 0},
         {2.80, 1.2496, -0.11921, 0.031130, -0.0093272, 0.0025161, 0},
         {2.62, 1.2568, -0.12573, 0.036423, -0.013132, 0.0047484, -0.0015979}},
        {{15.8, 1.0100, 0, 0, 0, 0, 0}, {4.80, 1.1640, -0.057991, 0, 0, 0, 0},
         {3.39, 1.2192, -0.094070, 0.014608, 0, 0, 0}, {2.90, 1.2422, -0.11269, 0.026140, -0.0064054, 0, 0},
         {2.65, 1.2534, -0.12257, 0.033755, -0.011081, 0.0036784, 0},
         {2.51, 1.2596, -0.12825, 0.038550, -0.014763, 0.0058619, -0.0024538}},
        {{9.16, 1.0300, 0, 0, 0, 0, 0}, {3.47, 1.1876, -0.072518, 0, 0, 0, 0},
         {2.91, 1.2341, -0.10569, 0.022589, 0, 0, 0}, {2.61, 1.2516, -0.12085, 0.032236, -0.011459, 0, 0},
         {2.45, 1.2596, -0.12829, 0.038533, -0.014681, 0.0072580, 0},
         {2.36, 1.2640, -0.13239, 0.042217, -0.017803, 0.0081959, -0.0051848}}};
    /* the reference stores the table as float; the double oracle keeps the
       same float-rounded coefficients so both solve the same discrete scheme */
    for (int k = 0; k <= 6; k++) c->hc[k] = (float)tab[c->maxrel][c->R - 1][k];
}

/* PML_pro.c:65-290 for one frame point: damping profile, then a and b */
static void FN(or_pml_point)(CTX *c, REAL *d, REAL *K, REAL *al, REAL *a, REAL *b, REAL d0, REAL ab, REAL thick,
                             const REAL alpha_max, int clamp)
{
    if (ab >= 0.0) {
        REAL an = ab / thick;
        *d = d0 * pow(an, c->npower);
        *K = 1.0 + (c->kmax - 1.0) * pow(an, c->npower);
        *al = alpha_max * (1.0 - an);
    }
    if (clamp && *al < 0.0) *al = 0.0;
    *b = exp(-(*d / *K + *al) * c->dt);
    if (abs((int)*d) > 1.0e-6) *a = *d * (*b - 1.0) / (*K * (*d + *K * *al));
}

static void FN(or_pml)(CTX *c)
{
    const int FW = c->fw;
    const REAL alpha_max = 2.0 * 3.141592653589793 * (c->fpml / 2.0);
    REAL thick = FW * c->dh;
    REAL Rcoef = 0.001;
    REAL d0 = -(c->npower + 1) * c->damping * log(Rcoef) / (2.0 * thick);
    REAL xl = thick, xr = (c->nx - 1) * c->dh - thick, yt = thick, yb = (c->ny - 1) * c->dh - thick;
    for (int i = 1; i <= FW; i++) {
        c->K_x[i] = c->K_xh[i] = c->K_y[i] = c->K_yh[i] = 1.0;
        REAL v = c->dh * (i - 1);
        FN(or_pml_point)(c, &c->d_x[i], &c->K_x[i], &c->al_x[i], &c->a_x[i], &c->b_x[i], d0, xl - v, thick, alpha_max, 1);
        FN(or_pml_point)(c, &c->d_xh[i], &c->K_xh[i], &c->al_xh[i], &c->a_xh[i], &c->b_xh[i], d0,
                         (REAL)(xl - (v + c->dh / 2.0)), thick, alpha_max, 1);
        FN(or_pml_point)(c, &c->d_y[i], &c->K_y[i], &c->al_y[i], &c->a_y[i], &c->b_y[i], d0, yt - v, thick, alpha_max, 0);
        FN(or_pml_point)(c, &c->d_yh[i], &c->K_yh[i], &c->al_yh[i], &c->a_yh[i], &c->b_yh[i], d0,
                         (REAL)(yt - (v + c->dh / 2.0)), thick, alpha_max, 0);
    }
    for (int i = c->nx - FW + 1; i <= c->nx; i++) {
        int h = i - c->nx + 2 * FW;
        c->K_x[h] = c->K_xh[h] = 1.0;
        REAL v = c->dh * (i - 1);
        FN(or_pml_point)(c, &c->d_x[h], &c->K_x[h], &c->al_x[h], &c->a_x[h], &c->b_x[h], d0, v - xr, thick, alpha_max, 1);
        FN(or_pml_point)(c, &c->d_xh[h], &c->K_xh[h], &c->al_xh[h], &c->a_xh[h], &c->b_xh[h], d0,
                         (REAL)(v + c->dh / 2.0 - xr), thick, alpha_max, 1);
    }
    for (int i = c->ny - FW + 1; i <= c->ny; i++) {
        int h = i - c->ny + 2 * FW;
        c->K_y[h] = c->K_yh[h] = 1.0;
        REAL v = c->dh * (i - 1);
        FN(or_pml_point)(c, &c->d_y[h], &c->K_y[h], &c->al_y[h], &c->a_y[h], &c->b_y[h], d0, v - yb, thick, alpha_max, 0);
        FN(or_pml_point)(c, &c->d_yh[h], &c->K_yh[h], &c->al_yh[h], &c->a_yh[h], &c->b_yh[h], d0,
                         (REAL)(v + c->dh / 2.0 - yb), thick, alpha_max, 0);
    }
}

/* matcopy_*_PSV on one rank: rows 0 / NY+1 from the opposite edge, then columns */
static void FN(or_wrap)(CTX *c, REAL *a)
{
    for (int i = 0; i <= c->nx + 1; i++) {
        REAL top = AT(a, 1, i), bot = AT(a, c->ny, i);
        AT(a, c->ny + 1, i) = top;
        AT(a, 0, i) = bot;
    }
    for (int j = 0; j <= c->ny + 1; j++) {
        REAL l = AT(a, j, 1), r = AT(a, j, c->nx);
        AT(a, j, c->nx + 1) = l;
        AT(a, j, 0) = r;
    }
}

/* av_mue.c:29-44, av_rho.c:13-22, av_tau.c:13, readmod_visc_PSV.c:31-35,119-120,
 * prepare_update_s_visc_PSV.c:23-90 (INVMAT1 = 1) */
static void FN(or_materials)(CTX *c, const float *qp, const float *qs)
{
    const int nx = c->nx, ny = c->ny, L = c->L;
    FN(or_wrap)(c, c->rho);
    FN(or_wrap)(c, c->pi);
    FN(or_wrap)(c, c->u);
    if (L) {
        for (int i = 1; i <= nx; i++)
            for (int j = 1; j <= ny; j++) {
                REAL qsv = c->honor_q ? (REAL)qs[FO(i, j)] : (REAL)30.0;
                REAL qpv = c->honor_q ? (REAL)qp[FO(i, j)] : (REAL)30.0;
                AT(c->taus, j, i) = 2.0 / qsv;
                AT(c->taup, j, i) = 2.0 / qpv;
            }
        FN(or_wrap)(c, c->taus);
        FN(or_wrap)(c, c->taup);
    }
    for (int j = 1; j <= ny; j++)
        for (int i = 1; i <= nx; i++) {
            REAL u1 = AT(c->rho, j, i) * AT(c->u, j, i) * AT(c->u, j, i);
            REAL u2 = AT(c->rho, j, i + 1) * AT(c->u, j, i + 1) * AT(c->u, j, i + 1);
            REAL u3 = AT(c->rho, j + 1, i) * AT(c->u, j + 1, i) * AT(c->u, j + 1, i);
            REAL u4 = AT(c->rho, j + 1, i + 1) * AT(c->u, j + 1, i + 1) * AT(c->u, j + 1, i + 1);
            AT(c->uipjp, j, i) = 4.0 / ((1.0 / u1) + (1.0 / u2) + (1.0 / u3) + (1.0 / u4));
            if ((u1 == 0.0) || (u2 == 0.0) || (u3 == 0.0) || (u4 == 0.0)) AT(c->uipjp, j, i) = 0.0;
            AT(c->rjp, j, i) = 1.0 / (0.5 * (AT(c->rho, j, i) + AT(c->rho, j + 1, i)));
            AT(c->rip, j, i) = 1.0 / (0.5 * (AT(c->rho, j, i) + AT(c->rho, j, i + 1)));
            if ((AT(c->rho, j, i) < 1e-4) && (AT(c->rho, j + 1, i) < 1e-4)) AT(c->rjp, j, i) = 0.0;
            if ((AT(c->rho, j, i) < 1e-4) && (AT(c->rho, j, i + 1) < 1e-4)) AT(c->rip, j, i) = 0.0;
            if (L)
                AT(c->tausipjp, j, i) =
                    0.25 * (AT(c->taus, j, i) + AT(c->taus, j, i + 1) + AT(c->taus, j + 1, i) + AT(c->taus, j + 1, i + 1));
        }
    if (!L) return;
    REAL pts[6];
    for (int l = 1; l <= L; l++) {
        pts[l] = 1.0 / (2.0 * 3.141592653589793 * c->fl[l]);
        c->eta[l] = c->dt / pts[l];
    }
    REAL ws = 2.0 * 3.141592653589793 * c->fl[1];
    REAL sumu = 0.0, sumpi = 0.0;
    for (int l = 1; l <= L; l++) {
        sumu = sumu + ((ws * ws * pts[l] * pts[l]) / (1.0 + ws * ws * pts[l] * pts[l]));
        sumpi = sumpi + ((ws * ws * pts[l] * pts[l]) / (1.0 + ws * ws * pts[l] * pts[l]));
    }
    for (int l = 1; l <= L; l++) {
        c->bip[l] = 1.0 / (1.0 + (c->eta[l] * 0.5));
        c->bjm[l] = 1.0 / (1.0 + (c->eta[l] * 0.5));
        c->cip[l] = 1.0 - (c->eta[l] * 0.5);
        c->cjm[l] = 1.0 - (c->eta[l] * 0.5);
    }
    for (int j = 1; j <= ny; j++)
        for (int i = 1; i <= nx; i++) {
            REAL mu = (AT(c->u, j, i) * AT(c->u, j, i) * AT(c->rho, j, i)) / (1.0 + sumu * AT(c->taus, j, i));
            REAL pi = (AT(c->pi, j, i) * AT(c->pi, j, i) * AT(c->rho, j, i)) / (1.0 + sumpi * AT(c->taup, j, i));
            REAL muipjp = AT(c->uipjp, j, i) / (1.0 + sumu * AT(c->tausipjp, j, i));
            AT(c->fipjp, j, i) = muipjp * c->dt * (1.0 + L * AT(c->tausipjp, j, i));
            AT(c->f, j, i) = mu * c->dt * (1.0 + L * AT(c->taus, j, i));
            AT(c->g, j, i) = pi * c->dt * (1.0 + L * AT(c->taup, j, i));
            for (int l = 1; l <= L; l++) {
                AT(c->dip + (l - 1) * c->plane, j, i) = muipjp * c->eta[l] * AT(c->tausipjp, j, i);
                AT(c->d + (l - 1) * c->plane, j, i) = mu * c->eta[l] * AT(c->taus, j, i);
                AT(c->e + (l - 1) * c->plane, j, i) = pi * c->eta[l] * AT(c->taup, j, i);
            }
        }
}

CTX *FN(or_create)(const int *ip, const float *fp, const float *vp, const float *vs, const float *rho,
                   const float *qp, const float *qs, int nsrc, const int *src_i, const int *src_j,
                   const int *src_type, const float *src_azi, const float *signals, int ntr, const int *rec_i,
                   const int *rec_j)
{
    CTX *c = (CTX *)FN(or_zalloc)(1, sizeof(CTX));
    c->nx = ip[0];
    c->ny = ip[1];
    c->nt = ip[2];
    c->R = ip[3] / 2;
    c->maxrel = ip[4];
    c->free_surf = ip[5];
    c->fw = ip[6];
    c->L = ip[7];
    c->quelltypb = ip[8];
    c->dtinv = ip[9] > 0 ? ip[9] : 1;
    c->seismo = ip[10];
    c->eprecond = ip[11];
    c->honor_q = ip[12];
    c->dh = fp[0];
    c->dt = fp[1];
    c->damping = fp[2];
    c->fpml = fp[3];
    c->npower = fp[4];
    c->kmax = fp[5];
    c->ts = fp[6];
    for (int l = 1; l <= c->L; l++) c->fl[l] = fp[6 + l];
    FN(or_hc)(c);
    c->pitch = c->nx + 2 * H;
    c->rows = c->ny + 2 * H;
    c->plane = (size_t)c->pitch * c->rows;
    REAL **grids[] = {&c->vx, &c->vy, &c->sxx, &c->syy, &c->sxy, &c->vxp1, &c->vyp1, &c->rho, &c->pi, &c->u,
                      &c->rip, &c->rjp, &c->uipjp, &c->taus, &c->taup, &c->tausipjp, &c->fipjp, &c->f, &c->g};
    for (size_t k = 0; k < sizeof(grids) / sizeof(grids[0]); k++) *grids[k] = (REAL *)FN(or_zalloc)(c->plane, sizeof(REAL));
    int Lm = c->L > 0 ? c->L : 1;
    REAL **lgrids[] = {&c->r, &c->p, &c->q, &c->dip, &c->d, &c->e};
    for (int k = 0; k < 6; k++) *lgrids[k] = (REAL *)FN(or_zalloc)(c->plane * Lm, sizeof(REAL));
    size_t w = 2 * (size_t)c->fw + 1;
    REAL **vecs[] = {&c->K_x, &c->a_x, &c->b_x, &c->K_xh, &c->a_xh, &c->b_xh, &c->K_y, &c->a_y, &c->b_y, &c->K_yh,
                     &c->a_yh, &c->b_yh, &c->d_x, &c->al_x, &c->d_xh, &c->al_xh, &c->d_y, &c->al_y, &c->d_yh, &c->al_yh};
    for (int k = 0; k < 20; k++) *vecs[k] = (REAL *)FN(or_zalloc)(w, sizeof(REAL));
    REAL **xps[] = {&c->psi_sxx_x, &c->psi_sxy_x, &c->psi_vxx, &c->psi_vyx, &c->psi_vxxs};
    for (int k = 0; k < 5; k++) *xps[k] = (REAL *)FN(or_zalloc)((size_t)(c->ny + 1) * w, sizeof(REAL));
    REAL **zps[] = {&c->psi_syy_y, &c->psi_sxy_y, &c->psi_vyy, &c->psi_vxy};
    for (int k = 0; k < 4; k++) *zps[k] = (REAL *)FN(or_zalloc)(w * (c->nx + 1), sizeof(REAL));
    for (int i = 1; i <= c->nx; i++)
        for (int j = 1; j <= c->ny; j++) {
            AT(c->pi, j, i) = vp[FO(i, j)];
            AT(c->u, j, i) = vs[FO(i, j)];
            AT(c->rho, j, i) = rho[FO(i, j)];
        }
    if (c->fw > 0) FN(or_pml)(c);
    FN(or_materials)(c, qp, qs);
    c->nsrc = nsrc;
    c->ntr = ntr;
    c->src_i = (int *)FN(or_zalloc)(nsrc, sizeof(int));
    c->src_j = (int *)FN(or_zalloc)(nsrc, sizeof(int));
    c->src_type = (int *)FN(or_zalloc)(nsrc, sizeof(int));
    c->src_azi = (REAL *)FN(or_zalloc)(nsrc, sizeof(REAL));
    c->signals = (REAL *)FN(or_zalloc)((size_t)nsrc * (c->nt + 1), sizeof(REAL));
    for (int l = 0; l < nsrc; l++) {
        c->src_i[l] = src_i[l];
        c->src_j[l] = src_j[l];
        c->src_type[l] = src_type ? src_type[l] : 1;
        c->src_azi[l] = src_azi ? src_azi[l] : 0;
        for (int t = 1; t <= c->nt; t++) c->signals[(size_t)l * (c->nt + 1) + t] = signals[(size_t)l * c->nt + t - 1];
    }
    c->quelltyp = nsrc > 0 ? c->src_type[nsrc - 1] : 1;   /* update_v_PML_PSV.c:745 overwrite */
    c->rec_i = (int *)FN(or_zalloc)(ntr, sizeof(int));
    c->rec_j = (int *)FN(or_zalloc)(ntr, sizeof(int));
    for (int l = 0; l < ntr; l++) {
        c->rec_i[l] = rec_i[l];
        c->rec_j[l] = rec_j[l];
    }
    c->sec = (REAL *)FN(or_zalloc)((size_t)5 * ntr * (c->nt + 1), sizeof(REAL));
    for (int k = 0; k < 3; k++) c->res[k] = (REAL *)FN(or_zalloc)((size_t)ntr * (c->nt + 1), sizeof(REAL));
    size_t n = (size_t)c->nx * c->ny;
    REAL **accs[] = {&c->wc, &c->wcu, &c->wcr, &c->Ws, &c->Wr, &c->gvp, &c->gvs, &c->grho};
    for (int k = 0; k < 8; k++) *accs[k] = (REAL *)FN(or_zalloc)(n, sizeof(REAL));
    return c;
}

void FN(or_destroy)(CTX *c)
{
    if (!c) return;
    REAL *all[] = {c->vx, c->vy, c->sxx, c->syy, c->sxy, c->vxp1, c->vyp1, c->rho, c->pi, c->u, c->rip, c->rjp,
                   c->uipjp, c->taus, c->taup, c->tausipjp, c->fipjp, c->f, c->g, c->r, c->p, c->q, c->dip, c->d,
                   c->e, c->K_x, c->a_x, c->b_x, c->K_xh, c->a_xh, c->b_xh, c->K_y, c->a_y, c->b_y, c->K_yh, c->a_yh,
                   c->b_yh, c->d_x, c->al_x, c->d_xh, c->al_xh, c->d_y, c->al_y, c->d_yh, c->al_yh, c->psi_sxx_x,
                   c->psi_sxy_x, c->psi_vxx, c->psi_vyx, c->psi_vxxs, c->psi_syy_y, c->psi_sxy_y, c->psi_vyy,
                   c->psi_vxy, c->src_azi, c->signals, c->sec, c->res[0], c->res[1], c->res[2], c->snap, c->wc,
                   c->wcu, c->wcr, c->Ws, c->Wr, c->gvp, c->gvs, c->grho};
    for (size_t k = 0; k < sizeof(all) / sizeof(all[0]); k++) free(all[k]);
    free(c->src_i);
    free(c->src_j);
    free(c->src_type);
    free(c->rec_i);
    free(c->rec_j);
    free(c);
}

/* ---- time step ----------------------------------------------------------- */

/* update_v_PML_PSV.c:366-480 (any FDORDER, same sum order) and :738-768 */
static void FN(or_update_v)(CTX *c, int nt, int sw)
{
    const int R = c->R, nx = c->nx, ny = c->ny, FW = c->fw;
    const REAL *hc = c->hc;
#pragma omp parallel for schedule(static)
    for (int j = 1; j <= ny; j++)
        for (int i = 1; i <= nx; i++) {
            REAL sxx_x = hc[1] * (AT(c->sxx, j, i + 1) - AT(c->sxx, j, i));
            REAL sxy_x = hc[1] * (AT(c->sxy, j, i) - AT(c->sxy, j, i - 1));
            REAL sxy_y = hc[1] * (AT(c->sxy, j, i) - AT(c->sxy, j - 1, i));
            REAL syy_y = hc[1] * (AT(c->syy, j + 1, i) - AT(c->syy, j, i));
            for (int m = 2; m <= R; m++) {
                sxx_x = sxx_x + hc[m] * (AT(c->sxx, j, i + m) - AT(c->sxx, j, i - m + 1));
                sxy_x = sxy_x + hc[m] * (AT(c->sxy, j, i + m - 1) - AT(c->sxy, j, i - m));
                sxy_y = sxy_y + hc[m] * (AT(c->sxy, j + m - 1, i) - AT(c->sxy, j - m, i));
                syy_y = syy_y + hc[m] * (AT(c->syy, j + m, i) - AT(c->syy, j - m + 1, i));
            }
            if (FW > 0 && i <= FW) {
                XF(c->psi_sxx_x, j, i) = c->b_xh[i] * XF(c->psi_sxx_x, j, i) + c->a_xh[i] * sxx_x;
                sxx_x = sxx_x / c->K_xh[i] + XF(c->psi_sxx_x, j, i);
                XF(c->psi_sxy_x, j, i) = c->b_x[i] * XF(c->psi_sxy_x, j, i) + c->a_x[i] * sxy_x;
                sxy_x = sxy_x / c->K_x[i] + XF(c->psi_sxy_x, j, i);
            }
            if (FW > 0 && i >= nx - FW + 1) {
                int h = i - nx + 2 * FW;
                XF(c->psi_sxx_x, j, h) = c->b_xh[h] * XF(c->psi_sxx_x, j, h) + c->a_xh[h] * sxx_x;
                sxx_x = sxx_x / c->K_xh[h] + XF(c->psi_sxx_x, j, h);
                XF(c->psi_sxy_x, j, h) = c->b_x[h] * XF(c->psi_sxy_x, j, h) + c->a_x[h] * sxy_x;
                sxy_x = sxy_x / c->K_x[h] + XF(c->psi_sxy_x, j, h);
            }
            if (FW > 0 && !c->free_surf && j <= FW) {
                ZF(c->psi_syy_y, j, i) = c->b_yh[j] * ZF(c->psi_syy_y, j, i) + c->a_yh[j] * syy_y;
                syy_y = syy_y / c->K_yh[j] + ZF(c->psi_syy_y, j, i);
                ZF(c->psi_sxy_y, j, i) = c->b_y[j] * ZF(c->psi_sxy_y, j, i) + c->a_y[j] * sxy_y;
                sxy_y = sxy_y / c->K_y[j] + ZF(c->psi_sxy_y, j, i);
            }
            if (FW > 0 && j >= ny - FW + 1) {
                int h = j - ny + 2 * FW;
                ZF(c->psi_syy_y, h, i) = c->b_yh[h] * ZF(c->psi_syy_y, h, i) + c->a_yh[h] * syy_y;
                syy_y = syy_y / c->K_yh[h] + ZF(c->psi_syy_y, h, i);
                ZF(c->psi_sxy_y, h, i) = c->b_y[h] * ZF(c->psi_sxy_y, h, i) + c->a_y[h] * sxy_y;
                sxy_y = sxy_y / c->K_y[h] + ZF(c->psi_sxy_y, h, i);
            }
            if (sw == 0) {
                AT(c->vxp1, j, i) = AT(c->rip, j, i) * (sxx_x + sxy_y) / c->dh;
                AT(c->vyp1, j, i) = AT(c->rjp, j, i) * (sxy_x + syy_y) / c->dh;
            } else {
                AT(c->vxp1, j, i) += c->dt * AT(c->vx, j, i);
                AT(c->vyp1, j, i) += c->dt * AT(c->vy, j, i);
            }
            AT(c->vx, j, i) += c->dt * AT(c->rip, j, i) * (sxx_x + sxy_y) / c->dh;
            AT(c->vy, j, i) += c->dt * AT(c->rjp, j, i) * (sxy_x + syy_y) / c->dh;
        }
    if (sw == 0) {
        for (int l = 0; l < c->nsrc; l++) {
            int i = c->src_i[l], j = c->src_j[l];
            REAL azi_rad = c->src_azi[l] * 3.141592653589793 / 180;
            REAL s = c->signals[(size_t)l * (c->nt + 1) + nt];
            if (c->src_type[l] == 2) AT(c->vx, j, i) += s;
            if (c->src_type[l] == 3) AT(c->vy, j, i) += s;
            if (c->src_type[l] == 4) {
                AT(c->vx, j, i) += -sin(azi_rad) * s;
                AT(c->vy, j, i) += cos(azi_rad) * s;
            }
        }
    } else {
        const int q = c->quelltypb;
        for (int l = 0; l < c->ntr; l++) {
            int i = c->rec_i[l], j = c->rec_j[l];
            REAL rx = c->res[0][(size_t)l * (c->nt + 1) + nt], ry = c->res[1][(size_t)l * (c->nt + 1) + nt];
            if (q == 1) {
                AT(c->vx, j, i) += rx;
                AT(c->vy, j, i) += ry;
            }
            if (q == 2 || q == 6 || q == 7) AT(c->vy, j, i) += ry;
            if (q == 3 || q == 5 || q == 7) AT(c->vx, j, i) += rx;
        }
    }
}

/* the four velocity derivatives of update_s_*_PML_PSV.c with CPML (case 8 = :366-438) */
static void FN(or_vderiv)(CTX *c, int j, int i, REAL dhi, REAL *pvxx, REAL *pvyx, REAL *pvxy, REAL *pvyy)
{
    const int R = c->R, nx = c->nx, ny = c->ny, FW = c->fw;
    const REAL *hc = c->hc;
    REAL vxx = hc[1] * (AT(c->vx, j, i) - AT(c->vx, j, i - 1));
    REAL vyx = hc[1] * (AT(c->vy, j, i + 1) - AT(c->vy, j, i));
    REAL vxy = hc[1] * (AT(c->vx, j + 1, i) - AT(c->vx, j, i));
    REAL vyy = hc[1] * (AT(c->vy, j, i) - AT(c->vy, j - 1, i));
    for (int m = 2; m <= R; m++) {
        vxx = vxx + hc[m] * (AT(c->vx, j, i + m - 1) - AT(c->vx, j, i - m));
        vyx = vyx + hc[m] * (AT(c->vy, j, i + m) - AT(c->vy, j, i - m + 1));
        vxy = vxy + hc[m] * (AT(c->vx, j + m, i) - AT(c->vx, j - m + 1, i));
        vyy = vyy + hc[m] * (AT(c->vy, j + m - 1, i) - AT(c->vy, j - m, i));
    }
    vxx = vxx * dhi;
    vyx = vyx * dhi;
    vxy = vxy * dhi;
    vyy = vyy * dhi;
    if (FW > 0 && i <= FW) {
        XF(c->psi_vxx, j, i) = c->b_x[i] * XF(c->psi_vxx, j, i) + c->a_x[i] * vxx;
        vxx = vxx / c->K_x[i] + XF(c->psi_vxx, j, i);
        XF(c->psi_vyx, j, i) = c->b_xh[i] * XF(c->psi_vyx, j, i) + c->a_xh[i] * vyx;
        vyx = vyx / c->K_xh[i] + XF(c->psi_vyx, j, i);
    }
    if (FW > 0 && i >= nx - FW + 1) {
        int h = i - nx + 2 * FW;
        XF(c->psi_vxx, j, h) = c->b_x[h] * XF(c->psi_vxx, j, h) + c->a_x[h] * vxx;
        vxx = vxx / c->K_x[h] + XF(c->psi_vxx, j, h);
        XF(c->psi_vyx, j, h) = c->b_xh[h] * XF(c->psi_vyx, j, h) + c->a_xh[h] * vyx;
        vyx = vyx / c->K_xh[h] + XF(c->psi_vyx, j, h);
    }
    if (FW > 0 && !c->free_surf && j <= FW) {
        ZF(c->psi_vyy, j, i) = c->b_y[j] * ZF(c->psi_vyy, j, i) + c->a_y[j] * vyy;
        ZF(c->psi_vxy, j, i) = c->b_yh[j] * ZF(c->psi_vxy, j, i) + c->a_yh[j] * vxy;
        vyy = vyy / c->K_y[j] + ZF(c->psi_vyy, j, i);
        vxy = vxy / c->K_yh[j] + ZF(c->psi_vxy, j, i);
    }
    if (FW > 0 && j >= ny - FW + 1) {
        int h = j - ny + 2 * FW;
        ZF(c->psi_vyy, h, i) = c->b_y[h] * ZF(c->psi_vyy, h, i) + c->a_y[h] * vyy;
        vyy = vyy / c->K_y[h] + ZF(c->psi_vyy, h, i);
        ZF(c->psi_vxy, h, i) = c->b_yh[h] * ZF(c->psi_vxy, h, i) + c->a_yh[h] * vxy;
        vxy = vxy / c->K_yh[h] + ZF(c->psi_vxy, h, i);
    }
    *pvxx = vxx;
    *pvyx = vyx;
    *pvxy = vxy;
    *pvyy = vyy;
}

/* update_s_elastic_PML_PSV.c:440-456 (INVMAT1 1) */
static void FN(or_update_s_el)(CTX *c)
{
    REAL dhi = c->dt / c->dh;
#pragma omp parallel for schedule(static)
    for (int j = 1; j <= c->ny; j++)
        for (int i = 1; i <= c->nx; i++) {
            REAL vxx, vyx, vxy, vyy;
            FN(or_vderiv)(c, j, i, dhi, &vxx, &vyx, &vxy, &vyy);
            REAL fipjp = AT(c->uipjp, j, i);
            REAL f = AT(c->rho, j, i) * AT(c->u, j, i) * AT(c->u, j, i);
            REAL g = AT(c->rho, j, i) * ((AT(c->pi, j, i) * AT(c->pi, j, i)) - 2 * AT(c->u, j, i) * AT(c->u, j, i));
            AT(c->sxy, j, i) += fipjp * (vyx + vxy);
            AT(c->sxx, j, i) += g * (vxx + vyy) + (2.0 * f * vxx);
            AT(c->syy, j, i) += g * (vxx + vyy) + (2.0 * f * vyy);
        }
}

/* update_s_visc_PML_PSV.c:440-501 */
static void FN(or_update_s_vi)(CTX *c)
{
    const int L = c->L;
    REAL dhi = 1.0 / c->dh;
    REAL dthalbe = c->dt / 2.0;
#pragma omp parallel for schedule(static)
    for (int j = 1; j <= c->ny; j++)
        for (int i = 1; i <= c->nx; i++) {
            REAL vxx, vyx, vxy, vyy;
            FN(or_vderiv)(c, j, i, dhi, &vxx, &vyx, &vxy, &vyy);
            REAL sumr = 0.0, sump = 0.0, sumq = 0.0;
            for (int l = 0; l < L; l++) {
                sumr += AT(c->r + l * c->plane, j, i);
                sump += AT(c->p + l * c->plane, j, i);
                sumq += AT(c->q + l * c->plane, j, i);
            }
            AT(c->sxy, j, i) += (AT(c->fipjp, j, i) * (vxy + vyx)) + (dthalbe * sumr);
            AT(c->sxx, j, i) += (AT(c->g, j, i) * (vxx + vyy)) - (2.0 * AT(c->f, j, i) * vyy) + (dthalbe * sump);
            AT(c->syy, j, i) += (AT(c->g, j, i) * (vxx + vyy)) - (2.0 * AT(c->f, j, i) * vxx) + (dthalbe * sumq);
            sumr = sump = sumq = 0.0;
            for (int l = 0; l < L; l++) {
                REAL *r = &AT(c->r + l * c->plane, j, i), *p = &AT(c->p + l * c->plane, j, i);
                REAL *q = &AT(c->q + l * c->plane, j, i);
                REAL dip = AT(c->dip + l * c->plane, j, i), d = AT(c->d + l * c->plane, j, i);
                REAL e = AT(c->e + l * c->plane, j, i);
                *r = c->bip[l + 1] * (*r * c->cip[l + 1] - (dip * (vxy + vyx)));
                *p = c->bjm[l + 1] * (*p * c->cjm[l + 1] - (e * (vxx + vyy)) + (2.0 * d * vyy));
                *q = c->bjm[l + 1] * (*q * c->cjm[l + 1] - (e * (vxx + vyy)) + (2.0 * d * vxx));
                sumr += *r;
                sump += *p;
                sumq += *q;
            }
            AT(c->sxy, j, i) += (dthalbe * sumr);
            AT(c->sxx, j, i) += (dthalbe * sump);
            AT(c->syy, j, i) += (dthalbe * sumq);
        }
}

/* psource.c:23-53 and msource.c:27-41 */
static void FN(or_psource)(CTX *c, int nt, int sw)
{
    if (sw == 1) {
        if (c->quelltypb < 4) return;
        for (int l = 0; l < c->ntr; l++) {
            REAL s = c->res[2][(size_t)l * (c->nt + 1) + nt];
            AT(c->sxx, c->rec_j[l], c->rec_i[l]) += s;
            AT(c->syy, c->rec_j[l], c->rec_i[l]) += s;
        }
        return;
    }
    if (c->quelltyp != 1 && c->quelltyp != 5) return;
    for (int l = 0; l < c->nsrc; l++) {
        const REAL *sg = c->signals + (size_t)l * (c->nt + 1);
        REAL amp = 0.0;
        if (nt == 1) amp = sg[nt + 1] / c->dt;
        if ((nt > 1) && (nt < c->nt)) amp = (sg[nt + 1] - sg[nt - 1]) / c->dt;
        if (nt == c->nt) amp = -sg[nt - 1] / c->dt;
        int i = c->src_i[l], j = c->src_j[l];
        if (c->quelltyp == 1) {
            AT(c->sxx, j, i) += amp;
            AT(c->syy, j, i) += amp;
        } else {
            REAL M11 = 0.0, M12 = 1.0, M22 = 0.0;
            AT(c->sxx, j, i) += amp * M11;
            AT(c->syy, j, i) += amp * M22;
            AT(c->sxy, j, i) += 0.25 * amp * M12;
            AT(c->sxy, j, i - 1) += 0.25 * amp * M12;
            AT(c->sxy, j - 1, i) += 0.25 * amp * M12;
            AT(c->sxy, j - 1, i - 1) += 0.25 * amp * M12;
        }
    }
}

/* surface_elastic_PML_PSV.c:29-103 and surface_visc_PML_PSV.c:34-170 */
static void FN(or_surface)(CTX *c)
{
    const int j = 1, R = c->R, FW = c->fw, L = c->L;
    const REAL dh24 = 1.0 / c->dh, dthalbe = c->dt / 2.0;
    REAL sumu = 0.0, sumpi = 0.0;
    if (L) {
        REAL pts[6];
        for (int l = 1; l <= L; l++) pts[l] = 1.0 / (2.0 * 3.141592653589793 * c->fl[l]);
        REAL ws = 2.0 * 3.141592653589793 * (1.0 / c->ts);
        for (int l = 1; l <= L; l++) {
            sumu = sumu + ((ws * ws * pts[l] * pts[l]) / (1.0 + ws * ws * pts[l] * pts[l]));
            sumpi = sumpi + ((ws * ws * pts[l] * pts[l]) / (1.0 + ws * ws * pts[l] * pts[l]));
        }
    }
    for (int i = 1; i <= c->nx; i++) {
        AT(c->syy, j, i) = 0.0;
        for (int l = 0; l < L; l++) AT(c->q + l * c->plane, j, i) = 0.0;
        REAL vxx = 0.0, vyy = 0.0;
        for (int m = 1; m <= R; m++) {
            AT(c->syy, j - m, i) = -AT(c->syy, j + m, i);
            AT(c->sxy, j - m, i) = -AT(c->sxy, j + m - 1, i);
            vxx += c->hc[m] * (AT(c->vx, j, i + m - 1) - AT(c->vx, j, i - m));
            vyy += c->hc[m] * (AT(c->vy, j + m - 1, i) - AT(c->vy, j - m, i));
        }
        vxx *= dh24;
        vyy *= dh24;
        if (FW > 0 && i <= FW) {
            XF(c->psi_vxxs, j, i) = c->b_x[i] * XF(c->psi_vxxs, j, i) + c->a_x[i] * vxx;
            vxx = vxx / c->K_x[i] + XF(c->psi_vxxs, j, i);
        }
        if (FW > 0 && i >= c->nx - FW + 1) {
            int h = i - c->nx + 2 * FW;
            XF(c->psi_vxxs, j, h) = c->b_x[h] * XF(c->psi_vxxs, j, h) + c->a_x[h] * vxx;
            vxx = vxx / c->K_x[h] + XF(c->psi_vxxs, j, h);
        }
        if (!L) {
            REAL fjm = AT(c->rho, j, i) * AT(c->u, j, i) * AT(c->u, j, i) * 2.0;
            REAL g = AT(c->rho, j, i) * ((AT(c->pi, j, i) * AT(c->pi, j, i)) - 2 * AT(c->u, j, i) * AT(c->u, j, i));
            AT(c->sxx, j, i) += -c->dt * ((g * g) / (g + fjm) * vxx + g * vyy);
        } else {
            REAL mu = (AT(c->u, j, i) * AT(c->u, j, i) * AT(c->rho, j, i)) / (1.0 + sumu * AT(c->taus, j, i));
            REAL pi = (AT(c->pi, j, i) * AT(c->pi, j, i) * AT(c->rho, j, i)) / (1.0 + sumpi * AT(c->taup, j, i));
            REAL sump = 0.0;
            for (int l = 0; l < L; l++) sump += AT(c->p + l * c->plane, j, i);
            REAL fjm = mu * 2.0 * (1.0 + L * AT(c->taus, j, i));
            REAL g = pi * (1.0 + L * AT(c->taup, j, i));
            AT(c->sxx, j, i) += -(c->dt * (g - fjm) * (g - fjm) * vxx / g) - (c->dt * (g - fjm) * vyy) - (dthalbe * sump);
            sump = 0.0;
            for (int l = 1; l <= L; l++) {
                REAL bjm = c->eta[l] / (1.0 + (c->eta[l] * 0.5));
                REAL djm = 2.0 * mu * AT(c->taus, j, i);
                REAL e = pi * AT(c->taup, j, i);
                REAL *p = &AT(c->p + (l - 1) * c->plane, j, i);
                *p += bjm * (((djm - e) * ((fjm / g) - 1.0) * vxx) - ((djm - e) * vyy));
                sump += *p;
            }
            AT(c->sxx, j, i) += (dthalbe * sump);
        }
    }
}

/* seismo_ssg.c:24-105 */
static void FN(or_seismo)(CTX *c, int nt)
{
    const REAL dhi = c->dt / c->dh;
    for (int l = 0; l < c->ntr; l++) {
        int i = c->rec_i[l], j = c->rec_j[l];
        size_t k = (size_t)l * (c->nt + 1) + nt, S = (size_t)c->ntr * (c->nt + 1);
        if (c->seismo == 1 || c->seismo == 4) {
            c->sec[0 * S + k] = AT(c->vx, j, i);
            c->sec[1 * S + k] = AT(c->vy, j, i);
        }
        if (c->seismo == 2 || c->seismo == 4) c->sec[2 * S + k] = -AT(c->sxx, j, i) - AT(c->syy, j, i);
        if (c->seismo == 3 || c->seismo == 4) {
            REAL vxx = 0, vyy = 0, vyx = 0, vxy = 0;
            for (int m = 1; m <= c->R; m++) {
                vxx += c->hc[m] * (AT(c->vx, j, i + m - 1) - AT(c->vx, j, i - m));
                vyy += c->hc[m] * (AT(c->vy, j + m - 1, i) - AT(c->vy, j - m, i));
                vyx += c->hc[m] * (AT(c->vy, j, i + m) - AT(c->vy, j, i - m + 1));
                vxy += c->hc[m] * (AT(c->vx, j + m, i) - AT(c->vx, j - m + 1, i));
            }
            vxx *= dhi;
            vyy *= dhi;
            vyx *= dhi;
            vxy *= dhi;
            REAL muss = AT(c->u, j, i) * AT(c->u, j, i) * AT(c->rho, j, i);
            REAL lamss = AT(c->pi, j, i) * AT(c->pi, j, i) * AT(c->rho, j, i);
            c->sec[4 * S + k] = (vxx + vyy) * sqrt(lamss);
            c->sec[3 * S + k] = (vxy - vyx) * sqrt(muss);
        }
    }
}

/* psv.c:240-309: snapshot k of pvxp1, pvyp1, sxx, syy, sxy (GRAD_FORM 1) + eprecond */
static void FN(or_store)(CTX *c, int k)
{
    size_t n = (size_t)c->nx * c->ny;
    REAL *dst = c->snap + (size_t)k * 5 * n;
    REAL *src[5] = {c->vxp1, c->vyp1, c->sxx, c->syy, c->sxy};
#pragma omp parallel for schedule(static) collapse(2)
    for (int f = 0; f < 5; f++)
        for (int i = 1; i <= c->nx; i++)
            for (int j = 1; j <= c->ny; j++) dst[f * n + FO(i, j)] = AT(src[f], j, i);
    if (c->eprecond == 1 || c->eprecond == 3)
        for (int i = 1; i <= c->nx; i++)
            for (int j = 1; j <= c->ny; j++)
                c->Ws[FO(i, j)] += (AT(c->vx, j, i) * AT(c->vx, j, i)) + (AT(c->vy, j, i) * AT(c->vy, j, i));
}

/* psv.c:313-387 (GRAD_FORM 1, INVMAT1 1) */
static void FN(or_correlate)(CTX *c, int k)
{
    size_t n = (size_t)c->nx * c->ny;
    const REAL *s = c->snap + (size_t)k * 5 * n;
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= c->nx; i++)
        for (int j = 1; j <= c->ny; j++) {
            size_t o = FO(i, j);
            REAL frx = s[o], fry = s[n + o], fx = s[2 * n + o], fy = s[3 * n + o], fu = s[4 * n + o];
            REAL sxx = AT(c->sxx, j, i), syy = AT(c->syy, j, i), sxy = AT(c->sxy, j, i);
            c->wcr[o] += (AT(c->vxp1, j, i) * frx) + (AT(c->vyp1, j, i) * fry);
            c->wc[o] += (fx + fy) * (sxx + syy);
            REAL muss = AT(c->rho, j, i) * AT(c->u, j, i) * AT(c->u, j, i);
            REAL lamss = AT(c->rho, j, i) * AT(c->pi, j, i) * AT(c->pi, j, i) - 2.0 * muss;
            if (muss > 0.0)
                c->wcu[o] += ((1.0 / (muss * muss)) * (fu * sxy)) +
                             ((1.0 / 4.0) * ((fx + fy) * (sxx + syy)) / ((lamss + muss) * (lamss + muss))) +
                             ((1.0 / 4.0) * ((fx - fy) * (sxx - syy)) / (muss * muss));
            if (c->eprecond == 1) c->Wr[o] += (AT(c->vx, j, i) * AT(c->vx, j, i)) + (AT(c->vy, j, i) * AT(c->vy, j, i));
        }
}

/* ass_gradPSV.c:29-150 (INVMAT1 1, GRAD_FORM 1, iter 1) */
static void FN(or_ass_grad)(CTX *c)
{
    for (int i = 1; i <= c->nx; i++)
        for (int j = 1; j <= c->ny; j++) {
            size_t o = FO(i, j);
            REAL rho = AT(c->rho, j, i), pi = AT(c->pi, j, i), u = AT(c->u, j, i);
            REAL lam = -c->dt * c->wc[o];
            REAL muss = rho * u * u;
            REAL lamss = rho * pi * pi - 2.0 * muss;
            if ((muss > 0.0) || (lamss > 0.0)) lam = (1.0 / (4.0 * (lamss + muss) * (lamss + muss))) * lam;
            c->gvp[o] = 2.0 * pi * rho * lam;
            REAL mu = -c->dt * c->wcu[o];
            c->gvs[o] = (-4.0 * rho * u * lam) + 2.0 * rho * u * mu;
            REAL rho_s = -c->dt * c->wcr[o];
            c->grho[o] = (((pi * pi) - (2.0 * u * u)) * lam) + (u * u * mu) + rho_s;
        }
}

static void FN(or_zero)(CTX *c)
{
    REAL *g[] = {c->vx, c->vy, c->sxx, c->syy, c->sxy, c->vxp1, c->vyp1};
    for (int k = 0; k < 7; k++) memset(g[k], 0, c->plane * sizeof(REAL));
    int Lm = c->L > 0 ? c->L : 1;
    memset(c->r, 0, c->plane * Lm * sizeof(REAL));
    memset(c->p, 0, c->plane * Lm * sizeof(REAL));
    memset(c->q, 0, c->plane * Lm * sizeof(REAL));
    size_t w = 2 * (size_t)c->fw + 1;
    REAL *xps[] = {c->psi_sxx_x, c->psi_sxy_x, c->psi_vxx, c->psi_vyx, c->psi_vxxs};
    for (int k = 0; k < 5; k++) memset(xps[k], 0, (size_t)(c->ny + 1) * w * sizeof(REAL));
    REAL *zps[] = {c->psi_syy_y, c->psi_sxy_y, c->psi_vyy, c->psi_vxy};
    for (int k = 0; k < 4; k++) memset(zps[k], 0, w * (c->nx + 1) * sizeof(REAL));
}

static void FN(or_step)(CTX *c, int nt, int mode)
{
    FN(or_update_v)(c, nt, mode == 1);
    if (c->L) FN(or_update_s_vi)(c);
    else FN(or_update_s_el)(c);
    FN(or_psource)(c, nt, mode == 1);
    if (c->free_surf) FN(or_surface)(c);
    if (mode != 1 && c->seismo) FN(or_seismo)(c, nt);
}

/* psv() mode 0 (store != 0: snapshots every DTINV steps) or mode 2; stops after nt_stop steps */
int FN(or_forward)(CTX *c, int store, int nt_stop)
{
    if (nt_stop <= 0 || nt_stop > c->nt) nt_stop = c->nt;
    FN(or_zero)(c);
    size_t n = (size_t)c->nx * c->ny;
    if (store) {
        c->nsnap = (int)ceil((float)c->nt / (float)c->dtinv);
        free(c->snap);
        c->snap = (REAL *)FN(or_zalloc)((size_t)c->nsnap * 5 * n, sizeof(REAL));
        REAL *accs[] = {c->wc, c->wcu, c->wcr, c->Ws, c->Wr};
        for (int k = 0; k < 5; k++) memset(accs[k], 0, n * sizeof(REAL));
    }
    for (int nt = 1; nt <= nt_stop; nt++) {
        FN(or_step)(c, nt, store ? 0 : 2);
        if (store && (nt - 1) % c->dtinv == 0) FN(or_store)(c, (nt - 1) / c->dtinv);
        if (isnan(AT(c->vy, c->ny / 2, c->nx / 2))) return -3;
    }
    return 0;
}

int FN(or_adjoint)(CTX *c, const float *res_vx, const float *res_vy, const float *res_p)
{
    if (!c->snap) return -8;
    const float *src[3] = {res_vx, res_vy, res_p};
    for (int k = 0; k < 3; k++) {
        memset(c->res[k], 0, (size_t)c->ntr * (c->nt + 1) * sizeof(REAL));
        if (src[k])
            for (int l = 0; l < c->ntr; l++)
                for (int t = 1; t <= c->nt; t++)
                    c->res[k][(size_t)l * (c->nt + 1) + t] = src[k][(size_t)l * c->nt + t - 1];
    }
    FN(or_zero)(c);
    for (int nt = 1; nt <= c->nt; nt++) {
        FN(or_step)(c, nt, 1);
        int nf = c->nt - nt + 1;
        if ((nf - 1) % c->dtinv == 0 && (nf - 1) / c->dtinv < c->nsnap) FN(or_correlate)(c, (nf - 1) / c->dtinv);
    }
    FN(or_ass_grad)(c);
    return 0;
}

int FN(or_get_sections)(CTX *c, int comp, REAL *out)
{
    size_t S = (size_t)c->ntr * (c->nt + 1);
    for (int l = 0; l < c->ntr; l++)
        for (int t = 1; t <= c->nt; t++) out[(size_t)l * c->nt + t - 1] = c->sec[comp * S + (size_t)l * (c->nt + 1) + t];
    return 0;
}

/* field ids as dn_shot_get_field */
int FN(or_get_field)(CTX *c, int field, REAL *out)
{
    size_t n = (size_t)c->nx * c->ny;
    if (field <= 6) {
        REAL *g[] = {c->vx, c->vy, c->sxx, c->syy, c->sxy, c->vxp1, c->vyp1};
        for (int i = 1; i <= c->nx; i++)
            for (int j = 1; j <= c->ny; j++) out[FO(i, j)] = AT(g[field], j, i);
        return 0;
    }
    REAL *a[] = {c->wc, c->wcu, c->wcr, c->Ws, c->Wr};
    if (field > 11) return -1;
    memcpy(out, a[field - 7], n * sizeof(REAL));
    return 0;
}

int FN(or_get_gradient)(CTX *c, REAL *gvp, REAL *gvs, REAL *grho)
{
    size_t n = (size_t)c->nx * c->ny;
    memcpy(gvp, c->gvp, n * sizeof(REAL));
    memcpy(gvs, c->gvs, n * sizeof(REAL));
    memcpy(grho, c->grho, n * sizeof(REAL));
    return 0;
}

/* which: 0 hc[7]; 1 CPML (20 x 2FW in dn_pml order); 2 rip 3 rjp 4 uipjp (file order) */
int FN(or_get_setup)(CTX *c, int which, REAL *out)
{
    if (which == 0) {
        for (int k = 0; k < 7; k++) out[k] = c->hc[k];
        return 0;
    }
    if (which == 1) {
        REAL *v[20] = {c->d_x, c->K_x, c->al_x, c->a_x, c->b_x, c->d_xh, c->K_xh, c->al_xh, c->a_xh, c->b_xh,
                       c->d_y, c->K_y, c->al_y, c->a_y, c->b_y, c->d_yh, c->K_yh, c->al_yh, c->a_yh, c->b_yh};
        for (int k = 0; k < 20; k++)
            for (int h = 1; h <= 2 * c->fw; h++) out[k * 2 * c->fw + h - 1] = v[k][h];
        return 0;
    }
    REAL *g = which == 2 ? c->rip : which == 3 ? c->rjp : which == 4 ? c->uipjp : NULL;
    if (!g) return -1;
    for (int i = 1; i <= c->nx; i++)
        for (int j = 1; j <= c->ny; j++) out[FO(i, j)] = AT(g, j, i);
    return 0;
}

#undef CTX
#undef FN
#undef H
#undef AT
#undef XF
#undef ZF
#undef FO
