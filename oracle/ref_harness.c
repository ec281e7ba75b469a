/*
 * ORACLE / TEST INFRASTRUCTURE - never part of the product.
 *
 * Drives the reference DENISE P-SV code (compiled unmodified from its own
 * sources, see oracle/Makefile) for a single shot on a single rank, through
 * flat arrays that ctypes can pass.  The call sequence mirrors the reference's
 * drivers:
 *   set-up:   FD_PSV.c:68-250 (initproc, alloc_*, PML_pro, holbergcoeff,
 *             readmod_*_PSV, matcopy_*, av_mue, av_rho, av_tau,
 *             prepare_update_s_visc_PSV)
 *   one shot: grad_obj_psv.c:61-215 (init_grad, psv mode 0, residuals
 *             supplied by the caller, srcpos_loc_back from the receivers,
 *             psv mode 1, ass_gradPSV)
 * Arrays cross this interface in file order (x-major, z contiguous).
 */
#include "fd.h"

/* globals defined by the reference (include/globvar.h) */
extern int NX, NY, NXG, NYG, NT, FDORDER, MAXRELERROR, FREE_SURF, FW, BOUNDARY, L, QUELLTYPB, DTINV, SEISMO, NDT;
extern int EPRECOND, MODE, GRAD_FORM, INVMAT1, INV_STF, MYID, MYID_SHOT, NPROCX, NPROCY, NPROC, NP, NCOLORS, COLOR;
extern int IDX, IDY, IDXI, IDYI, NTDTINV, NXNYI, SNAP, READMOD, WRITEMOD, PHYSICS, QUELLTYP, LOG;
extern int INV_VP_ITER, INV_VS_ITER, INV_RHO_ITER, RUN_MULTIPLE_SHOTS, QUELLART, N_ORDER, LNORM, TIMEWIN, TRKILL;
extern int OFFSET_MUTE, TIMELAPSE, TIME_FILT, COMP_WEIGHT, POS[3];
extern float DH, DT, DAMPING, FPML, npower, k_max_PML, TS, *FL, TSNAP1, TSNAP2, TSNAPINC, TIME;
extern char MFILE[STRING_SIZE];
extern FILE *FP;

static struct wavePSV W;
static struct wavePSV_PML WP;
static struct matPSV M;
static struct fwiPSV FWI;
static struct mpiPSV MP;
static struct seisPSV S;
static struct seisPSVfwi SF;
static struct acq A;
static float *hc = NULL;
static float **Ws = NULL, **Wr = NULL, **We = NULL;
static int *DTINV_help = NULL;
static int g_ready = 0, g_ntr = 0, g_nsrc = 0;
static MPI_Request *req_send, *req_rec;

/* ip: nx ny nt fdorder maxrelerror free_surf fw L quelltypb dtinv seismo eprecond mode
 * fp: dh dt damping fpml npower k_max_pml ts fl[0..4] */
int refh_setup(const int *ip, const float *fp, const char *mfile)
{
    FP = stderr;
    NX = NXG = ip[0];
    NY = NYG = ip[1];
    NT = ip[2];
    FDORDER = ip[3];
    MAXRELERROR = ip[4];
    FREE_SURF = ip[5];
    FW = ip[6];
    L = ip[7];
    QUELLTYPB = ip[8];
    DTINV = ip[9] > 0 ? ip[9] : 1;
    SEISMO = ip[10];
    EPRECOND = ip[11];
    MODE = ip[12];
    DH = fp[0];
    DT = fp[1];
    DAMPING = fp[2];
    FPML = fp[3];
    npower = fp[4];
    k_max_PML = fp[5];
    TS = fp[6];
    TIME = NT * DT;
    FL = vector(1, L > 0 ? L : 1);
    for (int l = 1; l <= L; l++) FL[l] = fp[6 + l];
    BOUNDARY = 0;
    NDT = 1;
    GRAD_FORM = 1;
    INVMAT1 = 1;
    INV_STF = 0;
    MYID = MYID_SHOT = 0;
    NPROCX = NPROCY = 1;
    NPROC = NP = 1;
    NCOLORS = 1;
    COLOR = 0;
    IDX = IDY = IDXI = IDYI = 1;
    SNAP = 0;
    READMOD = 1;
    WRITEMOD = 0;
    PHYSICS = 1;
    LOG = 0;
    INV_VP_ITER = INV_VS_ITER = INV_RHO_ITER = 0;
    N_ORDER = 0;
    LNORM = 2;
    TIMEWIN = TRKILL = OFFSET_MUTE = TIMELAPSE = TIME_FILT = 0;
    strncpy(MFILE, mfile, STRING_SIZE - 1);

    initproc();
    NTDTINV = ceil((float)NT / (float)DTINV);   /* FD_PSV.c:82 */
    NXNYI = (NX / IDXI) * (NY / IDYI);
    req_send = (MPI_Request *)malloc(REQUEST_COUNT * sizeof(MPI_Request));
    req_rec = (MPI_Request *)malloc(REQUEST_COUNT * sizeof(MPI_Request));

    alloc_PSV(&W, &WP);
    if (FW > 0)
        PML_pro(WP.d_x, WP.K_x, WP.alpha_prime_x, WP.a_x, WP.b_x, WP.d_x_half, WP.K_x_half, WP.alpha_prime_x_half,
                WP.a_x_half, WP.b_x_half, WP.d_y, WP.K_y, WP.alpha_prime_y, WP.a_y, WP.b_y, WP.d_y_half, WP.K_y_half,
                WP.alpha_prime_y_half, WP.a_y_half, WP.b_y_half);
    alloc_matPSV(&M);
    alloc_mpiPSV(&MP);
    if (MODE > 0) alloc_fwiPSV(&FWI);
    hc = holbergcoeff();
    if (L) readmod_visc_PSV(M.prho, M.ppi, M.pu, M.ptaus, M.ptaup, M.peta);
    else readmod_elastic_PSV(M.prho, M.ppi, M.pu);
    if (L) matcopy_PSV(M.prho, M.ppi, M.pu, M.ptaus, M.ptaup);
    else matcopy_elastic_PSV(M.prho, M.ppi, M.pu);
    av_mue(M.pu, M.puipjp, M.prho);
    av_rho(M.prho, M.prip, M.prjp);
    if (L) av_tau(M.ptaus, M.ptausipjp);
    if (L)
        prepare_update_s_visc_PSV(M.etajm, M.etaip, M.peta, M.fipjp, M.pu, M.puipjp, M.ppi, M.prho, M.ptaus, M.ptaup,
                                  M.ptausipjp, M.f, M.g, M.bip, M.bjm, M.cip, M.cjm, M.dip, M.d, M.e);
    Ws = matrix(1, NY, 1, NX);
    Wr = matrix(1, NY, 1, NX);
    We = matrix(1, NY, 1, NX);
    DTINV_help = ivector(1, NT);
    g_ready = 1;
    return 0;
}

int refh_get_hc(float *out)
{
    for (int k = 0; k <= 6; k++) out[k] = hc[k];
    return 0;
}

/* 20 vectors of 2*FW in dn_pml order: d K alpha a b for x, x_half, y, y_half */
int refh_get_pml(float *out)
{
    float *v[20] = {WP.d_x, WP.K_x, WP.alpha_prime_x, WP.a_x, WP.b_x, WP.d_x_half, WP.K_x_half,
                    WP.alpha_prime_x_half, WP.a_x_half, WP.b_x_half, WP.d_y, WP.K_y, WP.alpha_prime_y, WP.a_y,
                    WP.b_y, WP.d_y_half, WP.K_y_half, WP.alpha_prime_y_half, WP.a_y_half, WP.b_y_half};
    for (int k = 0; k < 20; k++)
        for (int h = 1; h <= 2 * FW; h++) out[k * 2 * FW + h - 1] = v[k][h];
    return 0;
}

static void to_file(float **a, float *out)
{
    for (int i = 1; i <= NX; i++)
        for (int j = 1; j <= NY; j++) out[(size_t)(i - 1) * NY + (j - 1)] = a[j][i];
}

/* which: 0 rip 1 rjp 2 uipjp 3 fipjp 4 f 5 g 6 tausipjp 7 taus 8 taup,
 *        100+l dip[l] 200+l d[l] 300+l e[l] (l = 1..L) */
int refh_get_mat(int which, float *out)
{
    if (which == 0) to_file(M.prip, out);
    else if (which == 1) to_file(M.prjp, out);
    else if (which == 2) to_file(M.puipjp, out);
    else if (which >= 3 && which <= 8 && L) {
        float **a[6] = {M.fipjp, M.f, M.g, M.ptausipjp, M.ptaus, M.ptaup};
        to_file(a[which - 3], out);
    } else if (which > 100 && L) {
        float ***t = which < 200 ? M.dip : (which < 300 ? M.d : M.e);
        int l = which % 100;
        for (int i = 1; i <= NX; i++)
            for (int j = 1; j <= NY; j++) out[(size_t)(i - 1) * NY + (j - 1)] = t[j][i][l];
    } else return -1;
    return 0;
}

/* bip bjm cip cjm eta [L each] */
int refh_get_visc_vectors(float *out)
{
    for (int l = 1; l <= L; l++) {
        out[0 * L + l - 1] = M.bip[l];
        out[1 * L + l - 1] = M.bjm[l];
        out[2 * L + l - 1] = M.cip[l];
        out[3 * L + l - 1] = M.cjm[l];
        out[4 * L + l - 1] = M.peta[l];
    }
    return 0;
}

/* srcpos: 8 rows x nsrc (the reference's srcpos_loc[1..8][l] = i, j, 0, tshift, fc, amp, azimuth, type) */
int refh_set_acq(int nsrc, const float *srcpos, const float *signals, int ntr, const int *rec_i, const int *rec_j)
{
    g_nsrc = nsrc;
    g_ntr = ntr;
    A.srcpos_loc = matrix(1, 8, 1, nsrc > 0 ? nsrc : 1);
    for (int r = 1; r <= 8; r++)
        for (int l = 1; l <= nsrc; l++) A.srcpos_loc[r][l] = srcpos[(r - 1) * nsrc + (l - 1)];
    A.signals = fmatrix(1, nsrc > 0 ? nsrc : 1, 1, NT);
    for (int l = 1; l <= nsrc; l++)
        for (int t = 1; t <= NT; t++) A.signals[l][t] = signals[(size_t)(l - 1) * NT + (t - 1)];
    A.recpos_loc = imatrix(1, 3, 1, ntr > 0 ? ntr : 1);
    for (int l = 1; l <= ntr; l++) {
        A.recpos_loc[1][l] = rec_i[l - 1];
        A.recpos_loc[2][l] = rec_j[l - 1];
        A.recpos_loc[3][l] = l;
    }
    alloc_seisPSV(ntr, NT, &S);
    if (MODE > 0) alloc_seisPSVfwi(ntr, ntr, NT, &SF);
    QUELLTYP = nsrc > 0 ? (int)A.srcpos_loc[8][1] : 1;   /* FD_PSV.c:298 */
    return 0;
}

/* psv() over all NT steps in `mode`; for mode 0 with MODE > 0 the per-shot
 * accumulators are re-initialised first (grad_obj_psv.c:61-70). */
int refh_run(int mode)
{
    if (mode == 0 && MODE > 0) {
        init_grad(FWI.waveconv_shot);
        init_grad(FWI.waveconv_u_shot);
        init_grad(FWI.waveconv_rho_shot);
        if (EPRECOND == 1 || EPRECOND == 3) {
            init_grad(Ws);
            init_grad(Wr);
            init_grad(We);
        }
    }
    if (mode == 1) {
        A.srcpos_loc_back = matrix(1, 6, 1, g_ntr);
        for (int i = 1; i <= g_ntr; i++) {
            A.srcpos_loc_back[1][i] = A.recpos_loc[1][i];
            A.srcpos_loc_back[2][i] = A.recpos_loc[2][i];
        }
        psv(&W, &WP, &M, &FWI, &MP, &S, &SF, &A, hc, 1, 1, g_ntr, NT, g_ntr, Ws, Wr, 1, DTINV_help, 1, req_send,
            req_rec);
    } else {
        psv(&W, &WP, &M, &FWI, &MP, &S, &SF, &A, hc, 1, 1, g_nsrc, NT, g_ntr, Ws, Wr, 1, DTINV_help, mode,
            req_send, req_rec);
    }
    return 0;
}

/* comp 0 vx 1 vy 2 p 3 curl 4 div -> [ntr][nt] */
int refh_get_sections(int comp, float *out)
{
    float **sec = comp == 0 ? S.sectionvx : comp == 1 ? S.sectionvy : comp == 2 ? S.sectionp
                : comp == 3 ? S.sectioncurl : S.sectiondiv;
    if (!sec) return -1;
    for (int r = 1; r <= g_ntr; r++)
        for (int t = 1; t <= NT; t++) out[(size_t)(r - 1) * NT + (t - 1)] = sec[r][t];
    return 0;
}

/* adjoint sources [ntr][nt] (NULL leaves a component untouched) */
int refh_set_residuals(const float *vx, const float *vy, const float *p)
{
    for (int r = 1; r <= g_ntr; r++)
        for (int t = 1; t <= NT; t++) {
            size_t k = (size_t)(r - 1) * NT + (t - 1);
            if (vx && SF.sectionvxdiff) SF.sectionvxdiff[r][t] = vx[k];
            if (vy && SF.sectionvydiff) SF.sectionvydiff[r][t] = vy[k];
            if (p && SF.sectionpdiff) SF.sectionpdiff[r][t] = p[k];
        }
    return 0;
}

/* The reference's L2 residual (calc_res.c, LNORM 2): data/syn [ntr][nt] in,
 * time-reversed residual [ntr][nt] out, returns 0.5 sum r^2 (test shot). */
double refh_calc_res(const float *data, const float *syn, float *diff)
{
    float **d = matrix(1, g_ntr, 1, NT), **s = matrix(1, g_ntr, 1, NT);
    float **df = matrix(1, g_ntr, 1, NT), **dfo = matrix(1, g_ntr, 1, NT);
    int **recpos = imatrix(1, 3, 1, g_ntr);
    float **srcpos = matrix(1, 8, 1, 1);
    for (int r = 1; r <= g_ntr; r++) {
        recpos[1][r] = A.recpos_loc[1][r];
        recpos[2][r] = A.recpos_loc[2][r];
        recpos[3][r] = r;
        for (int t = 1; t <= NT; t++) {
            d[r][t] = data[(size_t)(r - 1) * NT + (t - 1)];
            s[r][t] = syn[(size_t)(r - 1) * NT + (t - 1)];
        }
    }
    COMP_WEIGHT = 0;
    double l2 = calc_res(d, s, df, dfo, g_ntr, NT, 2, 0.0, 0, 1, 1, g_ntr, recpos, A.recpos_loc, srcpos, 1, 1, 1);
    for (int r = 1; r <= g_ntr; r++)
        for (int t = 1; t <= NT; t++) diff[(size_t)(r - 1) * NT + (t - 1)] = df[r][t];
    free_matrix(d, 1, g_ntr, 1, NT);
    free_matrix(s, 1, g_ntr, 1, NT);
    free_matrix(df, 1, g_ntr, 1, NT);
    free_matrix(dfo, 1, g_ntr, 1, NT);
    free_imatrix(recpos, 1, 3, 1, g_ntr);
    free_matrix(srcpos, 1, 8, 1, 1);
    return l2;
}

/* field ids match dn_shot_get_field: 0 vx 1 vy 2 sxx 3 syy 4 sxy 5 vxp1 6 vyp1
 * 7 waveconv_shot 8 waveconv_u_shot 9 waveconv_rho_shot 10 Ws 11 Wr */
int refh_get_field(int field, float *out)
{
    float **a = NULL;
    switch (field) {
    case 0: a = W.pvx; break;
    case 1: a = W.pvy; break;
    case 2: a = W.psxx; break;
    case 3: a = W.psyy; break;
    case 4: a = W.psxy; break;
    case 5: a = W.pvxp1; break;
    case 6: a = W.pvyp1; break;
    case 7: a = FWI.waveconv_shot; break;
    case 8: a = FWI.waveconv_u_shot; break;
    case 9: a = FWI.waveconv_rho_shot; break;
    case 10: a = Ws; break;
    case 11: a = Wr; break;
    default: return -1;
    }
    if (!a) return -1;
    to_file(a, out);
    return 0;
}

/* snapshot k (0-based) of field f (0 rho_x 1 rho_y 2 x 3 y 4 u), file order */
int refh_get_snapshot(int k, int f, float *out)
{
    float *v = f == 0 ? FWI.forward_prop_rho_x : f == 1 ? FWI.forward_prop_rho_y : f == 2 ? FWI.forward_prop_x
             : f == 3 ? FWI.forward_prop_y : FWI.forward_prop_u;
    for (size_t c = 0; c < (size_t)NXNYI; c++) out[c] = v[(size_t)k * NXNYI + c + 1];
    return 0;
}

/* ass_gradPSV of the current shot followed by the stacking of grad_obj_psv.c:253-261
 * into zeroed stacks; returns vp, vs, rho gradients in file order */
int refh_ass_grad(float *gvp, float *gvs, float *grho)
{
    ass_gradPSV(&FWI, &M, 1);
    to_file(FWI.waveconv_shot, gvp);
    to_file(FWI.waveconv_u_shot, gvs);
    to_file(FWI.waveconv_rho_shot, grho);
    return 0;
}

/* wavelet() of the reference (wavelet.c) for one source: QUELLART, tshift, fc, amp */
extern int QUELLART, N_ORDER;
int refh_wavelet(int quellart, int n_order, float tshift, float fc, float amp, float *out)
{
    float **sp = matrix(1, 8, 1, 1);
    sp[4][1] = tshift;
    sp[5][1] = fc;
    sp[6][1] = amp;
    QUELLART = quellart;
    N_ORDER = n_order;
    float **sig = wavelet(sp, 1, 1);
    for (int t = 1; t <= NT; t++) out[t - 1] = sig[1][t];
    N_ORDER = 0;
    return 0;
}

/* ---- host I/O of the reference --------------------------------------------- */
extern char SOURCE_FILE[STRING_SIZE], REC_FILE[STRING_SIZE];
extern float REFREC[4];
extern int SRCREC, READREC, SEIS_FORMAT;

static FILE *null_log(void)
{
    static FILE *f = NULL;
    if (!f) f = fopen("/dev/null", "w");
    return f;
}

/* read_par() on a parameter file; exports the globals the path reads:
 * iv[0..15] = MODE PHYSICS NPROCX NPROCY FDORDER MAXRELERROR NX NY QUELLART SRCREC
 *             RUN_MULTIPLE_SHOTS L FREE_SURF FW BOUNDARY SEISMO
 * iv[16..21] = READREC NDT SEIS_FORMAT INVMAT1 GRAD_FORM QUELLTYPB, iv[22] = DTINV
 * fv[0..12] = DH TIME DT TS DAMPING FPML npower k_max_PML REFREC[1] REFREC[2] FL[1] FL[2] FL[3]
 * strs: 8 x 74 chars: SOURCE_FILE REC_FILE MFILE SEIS_FILE_VX SEIS_FILE_VY SEIS_FILE_P SIGNAL_FILE JACOBIAN */
extern int RUN_MULTIPLE_SHOTS, BOUNDARY, INVMAT1;
extern char SEIS_FILE_VX[STRING_SIZE], SEIS_FILE_VY[STRING_SIZE], SEIS_FILE_P[STRING_SIZE], SIGNAL_FILE[STRING_SIZE],
    JACOBIAN[STRING_SIZE];
int refh_read_par(const char *path, int *iv, float *fv, char *strs)
{
    FILE *f = fopen(path, "r");
    if (!f) return -1;
    if (!FL) FL = vector(1, 8);
    read_par(f);   /* closes f */
    const int I[23] = {MODE, PHYSICS, NPROCX, NPROCY, FDORDER, MAXRELERROR, NX, NY, QUELLART, SRCREC,
                       RUN_MULTIPLE_SHOTS, L, FREE_SURF, FW, BOUNDARY, SEISMO, READREC, NDT, SEIS_FORMAT,
                       INVMAT1, GRAD_FORM, QUELLTYPB, DTINV};
    for (int k = 0; k < 23; k++) iv[k] = I[k];
    const float F[10] = {DH, TIME, DT, TS, DAMPING, FPML, npower, k_max_PML, REFREC[1], REFREC[2]};
    for (int k = 0; k < 10; k++) fv[k] = F[k];
    for (int l = 1; l <= 3; l++) fv[9 + l] = l <= L ? FL[l] : 0.0f;
    const char *S[8] = {SOURCE_FILE, REC_FILE, MFILE, SEIS_FILE_VX, SEIS_FILE_VY, SEIS_FILE_P, SIGNAL_FILE, JACOBIAN};
    for (int k = 0; k < 8; k++) {
        strncpy(strs + 74 * k, S[k], 73);
        strs[74 * k + 73] = 0;
    }
    return 0;
}

/* sources() on a source file: srcpos[8][n] flattened as srcpos[l*8 + r-1], TS */
int refh_sources(const char *path, int *nsrc, float *srcpos, int cap, float *ts)
{
    FP = null_log();
    strncpy(SOURCE_FILE, path, STRING_SIZE - 1);
    SRCREC = 1;
    float **sp = sources(nsrc);
    for (int l = 1; l <= *nsrc && l <= cap; l++)
        for (int r = 1; r <= 8; r++) srcpos[(l - 1) * 8 + r - 1] = sp[r][l];
    *ts = TS;
    return 0;
}

/* receiver() with READREC = 1 on <base>.dat */
int refh_receivers(const char *base, float refx, float refy, float dh, int *ntr, int *ri, int *rj, int cap)
{
    strncpy(REC_FILE, base, STRING_SIZE - 1);
    READREC = 1;
    REFREC[1] = refx;
    REFREC[2] = refy;
    REFREC[3] = 0.0f;
    DH = dh;
    int **rp = receiver(null_log(), ntr, 1);
    for (int k = 1; k <= *ntr && k <= cap; k++) {
        ri[k - 1] = rp[1][k];
        rj[k - 1] = rp[2][k];
    }
    return 0;
}

/* outseis_glob() SEIS_FORMAT 1 of a section [ntr][ns] (ns = NT samples) */
int refh_outseis_fmt(const char *path, int format, const float *section, int ntr, int ns, const int *ri,
                     const int *rj, float xs, float ys, int ndt, float time, float dt, float dh, float refx,
                     float refy);
int refh_outseis(const char *path, const float *section, int ntr, int ns, const int *ri, const int *rj, float xs,
                 float ys, int ndt, float time, float dt, float dh, float refx, float refy)
{
    return refh_outseis_fmt(path, 1, section, ntr, ns, ri, rj, xs, ys, ndt, time, dt, dh, refx, refy);
}

/* outseis_glob() with SEIS_FORMAT `format` (1 SU, 2 ASCII, 3 binary), as saveseis_glob.c calls it */
int refh_outseis_fmt(const char *path, int format, const float *section, int ntr, int ns, const int *ri,
                     const int *rj, float xs, float ys, int ndt, float time, float dt, float dh, float refx,
                     float refy)
{
    float **sec = matrix(1, ntr, 1, ns);
    int **rp = imatrix(1, 3, 1, ntr);
    float **sp = matrix(1, 8, 1, 1);
    for (int k = 1; k <= ntr; k++) {
        for (int t = 1; t <= ns; t++) sec[k][t] = section[(size_t)(k - 1) * ns + t - 1];
        rp[1][k] = ri[k - 1];
        rp[2][k] = rj[k - 1];
        rp[3][k] = 0;
    }
    sp[1][1] = xs;
    sp[2][1] = ys;
    NDT = ndt;
    TIME = time;
    DT = dt;
    DH = dh;
    REFREC[1] = refx;
    REFREC[2] = refy;
    FILE *f = fopen(path, "w");
    if (!f) return -1;
    outseis_glob(null_log(), f, 1, sec, rp, rp, ntr, sp, 1, ns, format, 1, 1);
    free_matrix(sec, 1, ntr, 1, ns);
    free_imatrix(rp, 1, 3, 1, ntr);
    free_matrix(sp, 1, 8, 1, 1);
    return 0;
}

/* ---- FWI outer loop of the reference ---------------------------------------- */
extern float EPSILON, EPSILON_u, EPSILON_rho, SCALERHO;
extern float VPUPPERLIM, VPLOWERLIM, VSUPPERLIM, VSLOWERLIM, RHOUPPERLIM, RHOLOWERLIM;

/* calc_opt_step() on three (step, misfit) pairs, 0-based in, the reference's 1-based inside */
float refh_calc_opt_step(const double *L2t3, const float *epst3)
{
    double L[4] = {0.0, L2t3[0], L2t3[1], L2t3[2]};
    float e[4] = {0.0f, epst3[0], epst3[1], epst3[2]};
    return calc_opt_step(L, e, 1);
}

/* calc_mat_change_test_PSV(itest = 1): arrays in file order */
int refh_mat_change(int nx, int ny, const float *vp, const float *vs, const float *rho, const float *gvp,
                    const float *gvs, const float *grho, float eps_scale, const float *lim, int iter,
                    const int *inv_iter, float scalerho, float *vp_out, float *vs_out, float *rho_out, float *eps3)
{
    NX = nx;
    NY = ny;
    MYID = 0;
    INVMAT1 = 1;
    VPLOWERLIM = lim[0];
    VPUPPERLIM = lim[1];
    VSLOWERLIM = lim[2];
    VSUPPERLIM = lim[3];
    RHOLOWERLIM = lim[4];
    RHOUPPERLIM = lim[5];
    INV_VP_ITER = inv_iter[0];
    INV_VS_ITER = inv_iter[1];
    INV_RHO_ITER = inv_iter[2];
    SCALERHO = scalerho;
    float **P = matrix(1, ny, 1, nx), **U = matrix(1, ny, 1, nx), **R = matrix(1, ny, 1, nx);
    float **Pn = matrix(1, ny, 1, nx), **Un = matrix(1, ny, 1, nx), **Rn = matrix(1, ny, 1, nx);
    float **Gp = matrix(1, ny, 1, nx), **Gu = matrix(1, ny, 1, nx), **Gr = matrix(1, ny, 1, nx);
    for (int i = 1; i <= nx; i++)
        for (int j = 1; j <= ny; j++) {
            const size_t o = (size_t)(i - 1) * ny + (j - 1);
            P[j][i] = vp[o];
            U[j][i] = vs[o];
            R[j][i] = rho[o];
            Gp[j][i] = gvp[o];
            Gu[j][i] = gvs[o];
            Gr[j][i] = grho[o];
        }
    calc_mat_change_test_PSV(Gp, Gr, Gu, R, Rn, P, Pn, U, Un, iter, 1, eps_scale, 1);
    for (int i = 1; i <= nx; i++)
        for (int j = 1; j <= ny; j++) {
            const size_t o = (size_t)(i - 1) * ny + (j - 1);
            vp_out[o] = Pn[j][i];
            vs_out[o] = Un[j][i];
            rho_out[o] = Rn[j][i];
        }
    eps3[0] = EPSILON;
    eps3[1] = EPSILON_u;
    eps3[2] = EPSILON_rho;
    free_matrix(P, 1, ny, 1, nx);
    free_matrix(U, 1, ny, 1, nx);
    free_matrix(R, 1, ny, 1, nx);
    free_matrix(Pn, 1, ny, 1, nx);
    free_matrix(Un, 1, ny, 1, nx);
    free_matrix(Rn, 1, ny, 1, nx);
    free_matrix(Gp, 1, ny, 1, nx);
    free_matrix(Gu, 1, ny, 1, nx);
    free_matrix(Gr, 1, ny, 1, nx);
    return 0;
}

/* ass_gradPSV followed by the per-shot energy preconditioning of
 * grad_obj_psv.c:218-240 (eprecond1 with the run's Ws/Wr; EPRECOND from set-up) */
extern float C_vp, C_vs, C_rho;
int refh_ass_grad_ep(const float *c3, float *gvp, float *gvs, float *grho)
{
    ass_gradPSV(&FWI, &M, 1);
    C_vp = c3[0];
    C_vs = c3[1];
    C_rho = c3[2];
    eprecond1(We, Ws, Wr);
    for (int i = 1; i <= NX; i++)
        for (int j = 1; j <= NY; j++) {
            FWI.waveconv_shot[j][i] = FWI.waveconv_shot[j][i] / (We[j][i] * C_vp * C_vp);
            FWI.waveconv_u_shot[j][i] = FWI.waveconv_u_shot[j][i] / (We[j][i] * C_vs * C_vs);
            if (C_vs == 0.0) FWI.waveconv_u_shot[j][i] = 0.0;
            FWI.waveconv_rho_shot[j][i] = FWI.waveconv_rho_shot[j][i] / (We[j][i] * C_rho * C_rho);
        }
    to_file(FWI.waveconv_shot, gvp);
    to_file(FWI.waveconv_u_shot, gvs);
    to_file(FWI.waveconv_rho_shot, grho);
    return 0;
}

/* ---- gradient conditioning of the reference --------------------------------- */
/* Globals of taper_grad.c, taper_grad_shot.c, smooth_grad.c and the filters it calls. */
extern int NXG, NYG, GRADT1, GRADT2, GRADT3, GRADT4, SWS_TAPER_GRAD_VERT, SWS_TAPER_GRAD_HOR;
extern int SWS_TAPER_GRAD_SOURCES, SWS_TAPER_FILE, SRTSHAPE, FILTSIZE, SPATFILTER;
extern float SRTRADIUS, EXP_TAPER_GRAD_HOR, WD_DAMP, WD_DAMP1, FC_END;
extern char TFILE[STRING_SIZE], JACOBIAN[STRING_SIZE];

/* Gradient arrays padded like the reference's waveconv (FWI_PSV.c allocates them with
 * the wavefield halo); taper_coeff gets a generous pad so that the source-box loops,
 * which may index a few cells left of column 1, stay inside the allocation. */
#define REFH_PAD 64
static float **grad_in(int nx, int ny, const float *a)
{
    float **m = matrix(-REFH_PAD, ny + REFH_PAD, -REFH_PAD, nx + REFH_PAD);
    for (int i = 1; i <= nx; i++)
        for (int j = 1; j <= ny; j++) m[j][i] = a[(size_t)(i - 1) * ny + (j - 1)];
    return m;
}
static void grad_out(int nx, int ny, float **m, float *a)
{
    for (int i = 1; i <= nx; i++)
        for (int j = 1; j <= ny; j++) a[(size_t)(i - 1) * ny + (j - 1)] = m[j][i];
    free_matrix(m, -REFH_PAD, ny + REFH_PAD, -REFH_PAD, nx + REFH_PAD);
}
static void precond_globals(int nx, int ny, float dh)
{
    NX = NXG = nx;
    NY = NYG = ny;
    DH = dh;
    MYID = 0;
    MYID_SHOT = 0;
    POS[1] = POS[2] = 0;
    NPROCX = NPROCY = 1;
    IDX = IDY = 1;
    FP = null_log();
}

/* precond_PSV (src/PSV/precond_PSV.c) on three gradients in file order.
 * sw = {vert, hor, sources, file}; srcxz = [nsrc][2] source x, z in metres;
 * tfile = the TFILE prefix (files tfile.bin, tfile_u.bin, tfile_rho.bin for sw[3]),
 * relative to the working directory, which must be writable (taper_grad writes
 * its coefficient files there). */
int refh_precond(int nx, int ny, float dh, const int *sw, const int *gradt, float exp_hor, int srtshape,
                 float srtradius, int filtsize, const char *tfile, int nsrc, const float *srcxz, int ntr,
                 const int *rec_i, const int *rec_j, float *g_vp, float *g_vs, float *g_rho)
{
    precond_globals(nx, ny, dh);
    SWS_TAPER_GRAD_VERT = sw[0];
    SWS_TAPER_GRAD_HOR = sw[1];
    SWS_TAPER_GRAD_SOURCES = sw[2];
    SWS_TAPER_FILE = sw[3];
    GRADT1 = gradt[0];
    GRADT2 = gradt[1];
    GRADT3 = gradt[2];
    GRADT4 = gradt[3];
    EXP_TAPER_GRAD_HOR = exp_hor;
    SRTSHAPE = srtshape;
    SRTRADIUS = srtradius;
    FILTSIZE = filtsize;
    snprintf(TFILE, STRING_SIZE, "%s", tfile);
    struct fwiPSV F;
    struct acq Q;
    memset(&F, 0, sizeof F);
    memset(&Q, 0, sizeof Q);
    F.waveconv = grad_in(nx, ny, g_vp);
    F.waveconv_u = grad_in(nx, ny, g_vs);
    F.waveconv_rho = grad_in(nx, ny, g_rho);
    Q.srcpos = matrix(1, 8, 1, nsrc > 0 ? nsrc : 1);
    for (int n = 1; n <= nsrc; n++) {
        Q.srcpos[1][n] = srcxz[2 * (n - 1)];
        Q.srcpos[2][n] = srcxz[2 * (n - 1) + 1];
    }
    Q.recpos = imatrix(1, 3, 1, ntr > 0 ? ntr : 1);
    for (int n = 1; n <= ntr; n++) {
        Q.recpos[1][n] = rec_i[n - 1];
        Q.recpos[2][n] = rec_j[n - 1];
    }
    float **tc = matrix(-REFH_PAD, ny + REFH_PAD, -REFH_PAD, nx + REFH_PAD);
    precond_PSV(&F, &Q, nsrc, ntr, tc, NULL);
    grad_out(nx, ny, F.waveconv, g_vp);
    grad_out(nx, ny, F.waveconv_u, g_vs);
    grad_out(nx, ny, F.waveconv_rho, g_rho);
    free_matrix(tc, -REFH_PAD, ny + REFH_PAD, -REFH_PAD, nx + REFH_PAD);
    free_matrix(Q.srcpos, 1, 8, 1, nsrc > 0 ? nsrc : 1);
    free_imatrix(Q.recpos, 1, 3, 1, ntr > 0 ? ntr : 1);
    return 0;
}

/* taper_grad_shot (src/taper_grad_shot.c) of shot ishot (1-based) on one gradient. */
int refh_taper_shot(int nx, int ny, float dh, int srtshape, float srtradius, int filtsize, const char *tfile,
                    int nsrc, const float *srcxz, int ishot, float *g)
{
    precond_globals(nx, ny, dh);
    SRTSHAPE = srtshape;
    SRTRADIUS = srtradius;
    FILTSIZE = filtsize;
    COLOR = 0;
    snprintf(TFILE, STRING_SIZE, "%s", tfile);
    float **srcpos = matrix(1, 8, 1, nsrc);
    for (int n = 1; n <= nsrc; n++) {
        srcpos[1][n] = srcxz[2 * (n - 1)];
        srcpos[2][n] = srcxz[2 * (n - 1) + 1];
    }
    int **recpos = imatrix(1, 3, 1, 1);
    float **w = grad_in(nx, ny, g);
    float **tc = matrix(-REFH_PAD, ny + REFH_PAD, -REFH_PAD, nx + REFH_PAD);
    taper_grad_shot(w, tc, srcpos, nsrc, recpos, 0, ishot);
    grad_out(nx, ny, w, g);
    free_matrix(tc, -REFH_PAD, ny + REFH_PAD, -REFH_PAD, nx + REFH_PAD);
    free_matrix(srcpos, 1, 8, 1, nsrc);
    free_imatrix(recpos, 1, 3, 1, 1);
    return 0;
}

/* smooth_grad (src/smooth_grad.c) on one gradient; vel = the S-velocity model
 * (file order) for SPATFILTER 4.  jacobian = the JACOBIAN prefix of the
 * temporary files, relative to the (writable) working directory. */
int refh_smooth_grad(int nx, int ny, float dh, int spatfilter, float wd_damp, float wd_damp1, float fc_end,
                     float c_vs, const char *jacobian, const float *vel, float *g)
{
    precond_globals(nx, ny, dh);
    SPATFILTER = spatfilter;
    WD_DAMP = wd_damp;
    WD_DAMP1 = wd_damp1;
    FC_END = fc_end;
    C_vs = c_vs;
    snprintf(JACOBIAN, STRING_SIZE, "%s", jacobian);
    float **w = grad_in(nx, ny, g);
    float **v = grad_in(nx, ny, vel);
    smooth_grad(w, v);
    grad_out(nx, ny, w, g);
    free_matrix(v, -REFH_PAD, ny + REFH_PAD, -REFH_PAD, nx + REFH_PAD);
    return 0;
}

/* calc_res (src/calc_res.c) with the options of the objective functions that
 * need no FFT.  iopt = {lnorm, grad_form, mode, n_order, comp_weight, trkill,
 * offset_mute, timewin}; fopt = {c_vp, c_rho, offsetc, gamma, twlength_minus,
 * fc_start, fc_end}; rec_i/rec_j grid indices, (src_x, src_z) metres;
 * killfile = the TRKILL_FILE (one row of ntr 0/1 flags) relative to the working
 * directory.  data/syn [ntr][ns] in, residual [ntr][ns] out; returns the misfit. */
extern int N_ORDER, OFFSET_MUTE, TIMEWIN, TRKILL;
extern float OFFSETC, GAMMA, TWLENGTH_MINUS, FC_START;
extern char TRKILL_FILE[STRING_SIZE];
double refh_calc_res_ex(int ntr, int ns, float dt, float dh, const int *iopt, const float *fopt, const int *rec_i,
                        const int *rec_j, float src_x, float src_z, const char *killfile, const float *data,
                        const float *syn, float *diff)
{
    MYID = 0;
    MYID_SHOT = 0;
    DT = dt;
    DH = dh;
    FP = null_log();
    GRAD_FORM = iopt[1];
    MODE = iopt[2];
    N_ORDER = iopt[3];
    COMP_WEIGHT = iopt[4];
    TRKILL = iopt[5];
    OFFSET_MUTE = iopt[6];
    TIMEWIN = iopt[7];
    C_vp = fopt[0];
    C_rho = fopt[1];
    OFFSETC = fopt[2];
    GAMMA = fopt[3];
    TWLENGTH_MINUS = fopt[4];
    FC_START = fopt[5];
    FC_END = fopt[6];
    snprintf(TRKILL_FILE, STRING_SIZE, "%s", killfile ? killfile : "");
    float **d = matrix(1, ntr, 1, ns), **s = matrix(1, ntr, 1, ns);
    float **df = matrix(1, ntr, 1, ns), **dfo = matrix(1, ntr, 1, ns);
    int **recpos = imatrix(1, 3, 1, ntr);
    float **srcpos = matrix(1, 8, 1, 1);
    srcpos[1][1] = src_x;
    srcpos[2][1] = src_z;
    for (int r = 1; r <= ntr; r++) {
        recpos[1][r] = rec_i[r - 1];
        recpos[2][r] = rec_j[r - 1];
        recpos[3][r] = r;
        for (int t = 1; t <= ns; t++) {
            d[r][t] = data[(size_t)(r - 1) * ns + (t - 1)];
            s[r][t] = syn[(size_t)(r - 1) * ns + (t - 1)];
        }
    }
    double l2 = calc_res(d, s, df, dfo, ntr, ns, iopt[0], 0.0, 0, 1, 1, ntr, recpos, recpos, srcpos, 1, 1, 1);
    for (int r = 1; r <= ntr; r++)
        for (int t = 1; t <= ns; t++) diff[(size_t)(r - 1) * ns + (t - 1)] = df[r][t];
    free_matrix(d, 1, ntr, 1, ns);
    free_matrix(s, 1, ntr, 1, ns);
    free_matrix(df, 1, ntr, 1, ns);
    free_matrix(dfo, 1, ntr, 1, ns);
    free_imatrix(recpos, 1, 3, 1, ntr);
    free_matrix(srcpos, 1, 8, 1, 1);
    return l2;
}

/* apply_tdfilt (src/apply_tdfilt.c) on [ntr][ns] traces in place. */
int refh_apply_tdfilt(int ntr, int ns, float dt, int order, float fc2, float fc1, float *data)
{
    DT = dt;
    float **s = matrix(1, ntr, 1, ns);
    for (int r = 1; r <= ntr; r++)
        for (int t = 1; t <= ns; t++) s[r][t] = data[(size_t)(r - 1) * ns + (t - 1)];
    apply_tdfilt(s, ntr, ns, order, fc2, fc1);
    for (int r = 1; r <= ntr; r++)
        for (int t = 1; t <= ns; t++) data[(size_t)(r - 1) * ns + (t - 1)] = s[r][t];
    free_matrix(s, 1, ntr, 1, ns);
    return 0;
}

/* read_par_inv (src/read_par_inv.c): stage nstage of a workflow file; out[30]
 * = PRO, TIME_FILT, FC_START, FC_END, ORDER, TIMEWIN, GAMMA, TWLENGTH_MINUS,
 * TWLENGTH_PLUS, INV_VP_ITER, INV_VS_ITER, INV_RHO_ITER, INV_QS_ITER,
 * SPATFILTER, WD_DAMP, WD_DAMP1, EPRECOND, LNORM, ROWI, INV_STF, OFFSETC_STF,
 * EPS_STF, NORMALIZE, OFFSET_MUTE, OFFSETC, SCALERHO, SCALEQS, ENV,
 * GAMMA_GRAV, N_ORDER (as doubles). */
extern int SPAT_FILT_SIZE, SPAT_FILT_1, SPAT_FILT_ITER, NORMALIZE, INV_QS_ITER, ENV, ORDER, ROWI;
extern float PRO, EPS_STF, OFFSETC_STF, TWLENGTH_PLUS, SCALEQS, GAMMA_GRAV;
int refh_read_par_inv(const char *path, int nstage, int stagemax, double *out)
{
    MYID = 1;   /* no banner */
    FILE *fp = fopen(path, "r");
    if (!fp) return -1;
    read_par_inv(fp, nstage, stagemax);
    const double v[30] = {PRO, TIME_FILT, FC_START, FC_END, ORDER, TIMEWIN, GAMMA, TWLENGTH_MINUS, TWLENGTH_PLUS,
                          INV_VP_ITER, INV_VS_ITER, INV_RHO_ITER, INV_QS_ITER, SPATFILTER, WD_DAMP, WD_DAMP1,
                          EPRECOND, LNORM, ROWI, INV_STF, OFFSETC_STF, EPS_STF, NORMALIZE, OFFSET_MUTE, OFFSETC,
                          SCALERHO, SCALEQS, ENV, GAMMA_GRAV, N_ORDER};
    for (int k = 0; k < 30; k++) out[k] = v[k];
    MYID = 0;
    return 0;
}

/* wavelet() of the reference for one source with every global it reads set here:
 * NT, DT, QUELLART, N_ORDER, FC_SPIKE_1, FC_SPIKE_2, TS and SIGNAL_FILE (QUELLART 3
 * reads "<signal_file>_shot_<ishot>.dat"); for QUELLART 6 the caller's
 * apply_tdfilt with ORDER_SPIKE, FC_SPIKE_2, FC_SPIKE_1 follows when filt > 0. */
extern float FC_SPIKE_1, FC_SPIKE_2;
int refh_wavelet_ex(int quellart, int n_order, int nt, float dt, float tshift, float fc, float amp, float fc_spike_1,
                    float fc_spike_2, float ts, const char *signal_file, int ishot, int filt_order, float *out)
{
    if (!FP) FP = null_log();   /* wavelet() logs to FP */
    float **sp = matrix(1, 8, 1, 1);
    sp[4][1] = tshift;
    sp[5][1] = fc;
    sp[6][1] = amp;
    NT = nt;
    DT = dt;
    QUELLART = quellart;
    N_ORDER = n_order;
    FC_SPIKE_1 = fc_spike_1;
    FC_SPIKE_2 = fc_spike_2;
    TS = ts;
    if (signal_file) snprintf(SIGNAL_FILE, STRING_SIZE, "%s", signal_file);
    float **sig = wavelet(sp, 1, ishot);
    if (quellart == 6 && filt_order > 0) apply_tdfilt(sig, 1, nt, filt_order, fc_spike_2, fc_spike_1);
    for (int t = 1; t <= nt; t++) out[t - 1] = sig[1][t];
    N_ORDER = 0;
    free_matrix(sig, 1, 1, 1, nt);
    free_matrix(sp, 1, 8, 1, 1);
    return 0;
}

/* read_par() lines 60-115 (inversion): iv[36] ints, fv[12] floats, strs 8 x 74 chars
 * (TFILE, INV_MODELFILE, TRKILL_FILE, PICKS_FILE, MISFIT_LOG_FILE, DATA_DIR_T0, DFILE, DATA_DIR) */
extern int ITERMAX, TAPER, TAPERLENGTH, TESTSHOT_START, TESTSHOT_END, TESTSHOT_INCR;
extern int SWS_TAPER_CIRCULAR_PER_SHOT, INV_MOD_OUT, GRAD_METHOD, NLBFGS, PCG_BETA, MODEL_FILTER, FILT_SIZE;
extern int STEPMAX, TRKILL, MIN_ITER, GRAD_FILTER, FILT_SIZE_GRAD, TIMELAPSE, RTMOD;
extern int GRAVITY, NZGRAV, NGRAVB, GRAV_TYPE, BACK_DENSITY, RTM_SHOT;
extern float EPS_SCALE, SCALEFAC, QSUPPERLIM, QSLOWERLIM;
extern char INV_MODELFILE[STRING_SIZE], PICKS_FILE[STRING_SIZE], MISFIT_LOG_FILE[STRING_SIZE];
extern char DATA_DIR_T0[STRING_SIZE], DFILE[STRING_SIZE], DATA_DIR[STRING_SIZE];
int refh_read_par_fwi(const char *path, int *iv, float *fv, char *strs)
{
    FILE *f = fopen(path, "r");
    if (!f) return -1;
    if (!FL) FL = vector(1, 8);
    read_par(f);   /* closes f */
    const int I[36] = {ITERMAX, TAPER, TAPERLENGTH, GRADT1, GRADT2, GRADT3, GRADT4, TESTSHOT_START, TESTSHOT_END,
                       TESTSHOT_INCR, SWS_TAPER_GRAD_VERT, SWS_TAPER_GRAD_HOR, SWS_TAPER_GRAD_SOURCES,
                       SWS_TAPER_CIRCULAR_PER_SHOT, SRTSHAPE, FILTSIZE, SWS_TAPER_FILE, INV_MOD_OUT, GRAD_METHOD,
                       PCG_BETA, NLBFGS, MODEL_FILTER, FILT_SIZE, STEPMAX, TRKILL, MIN_ITER, GRAD_FILTER,
                       FILT_SIZE_GRAD, TIMELAPSE, RTMOD, GRAVITY, NGRAVB, NZGRAV, GRAV_TYPE, BACK_DENSITY, RTM_SHOT};
    for (int k = 0; k < 36; k++) iv[k] = I[k];
    const float F[12] = {EXP_TAPER_GRAD_HOR, SRTRADIUS, VPUPPERLIM, VPLOWERLIM, VSUPPERLIM, VSLOWERLIM,
                         RHOUPPERLIM, RHOLOWERLIM, QSUPPERLIM, QSLOWERLIM, EPS_SCALE, SCALEFAC};
    for (int k = 0; k < 12; k++) fv[k] = F[k];
    const char *S[8] = {TFILE, INV_MODELFILE, TRKILL_FILE, PICKS_FILE, MISFIT_LOG_FILE, DATA_DIR_T0, DFILE, DATA_DIR};
    for (int k = 0; k < 8; k++) {
        strncpy(strs + 74 * k, S[k], 73);
        strs[74 * k + 73] = 0;
    }
    return 0;
}

/* ---- the reference's optimisers: FWI_PSV.c:637-676 -------------------------
 * GRAD_METHOD 2: the LBFGS_pointer rule of FWI_PSV.c:452-466, store_LBFGS_PSV,
 * LBFGS, extract_LBFGS_PSV (which keep the previous gradient and model in the
 * JACOBIAN files, here under `jacobian`); GRAD_METHOD 1: descent, store_PCG_PSV,
 * PCG, extract_PCG_PSV, store_PCG_PSV, descent.  Models and gradients cross in
 * file order; the gradients are replaced by the search direction.  The vectors
 * persist between calls like FWI_PSV.c's; refh_optim_reset is zero_LBFGS /
 * zero_PCG with LBFGS_pointer = 1 (FWI_PSV.c:800-811). */
static int o_method = 0, o_nlbfgs = 0, o_ptr = 1, o_vec = 0;
static float *o_y, *o_s, *o_q, *o_r, *o_rho, *o_alpha, *o_beta, *o_new, *o_old, *o_dir;

int refh_optim_init(int method, int nx, int ny, int nlbfgs, int pcg_beta, const char *jacobian)
{
    FP = stderr;
    NX = NXG = nx;
    NY = NYG = ny;
    IDX = IDY = 1;
    MYID = MYID_SHOT = 0;
    POS[1] = POS[2] = 0;
    NPROCX = NPROCY = 1;
    NPROC = NP = 1;
    PCG_BETA = pcg_beta;
    strncpy(JACOBIAN, jacobian, STRING_SIZE - 1);
    o_method = method;
    o_nlbfgs = nlbfgs;
    o_ptr = 1;
    o_vec = 3 * nx * ny;
    if (method == 2) {
        o_y = vector(1, o_vec * nlbfgs);
        o_s = vector(1, o_vec * nlbfgs);
        o_q = vector(1, o_vec);
        o_r = vector(1, o_vec);
        o_rho = vector(1, nlbfgs);
        o_alpha = vector(1, nlbfgs);
        o_beta = vector(1, nlbfgs);
    } else {
        o_old = vector(1, o_vec);
        o_new = vector(1, o_vec);
        o_dir = vector(1, o_vec);
    }
    return 0;
}

int refh_optim_reset(void)
{
    if (o_method == 2) {
        zero_LBFGS(o_nlbfgs, o_vec, o_y, o_s, o_q, o_r, o_alpha, o_beta, o_rho);
        o_ptr = 1;
    } else {
        zero_PCG(o_old, o_new, o_dir, o_vec);
    }
    return 0;
}

int refh_optim_step(int iter, const float *c3, const float *vp, const float *vs, const float *rho, float *gvp,
                    float *gvs, float *grho)
{
    const int nx = NX, ny = NY;
    C_vp = c3[0];
    C_vs = c3[1];
    C_rho = c3[2];
    float **P = grad_in(nx, ny, vp), **U = grad_in(nx, ny, vs), **R = grad_in(nx, ny, rho);
    float **G = grad_in(nx, ny, gvp), **Gu = grad_in(nx, ny, gvs), **Gr = grad_in(nx, ny, grho);
    float **Gp = grad_in(nx, ny, gvp), **Gpu = grad_in(nx, ny, gvs), **Gpr = grad_in(nx, ny, grho);
    if (o_method == 2) {
        if (iter > 2) o_ptr++;
        if (o_ptr > o_nlbfgs) o_ptr = 1;
        store_LBFGS_PSV(NULL, 0, NULL, NULL, 0, iter, G, Gp, Gu, Gpu, Gr, Gpr, o_y, o_s, o_q, P, U, R, nx * ny,
                        o_ptr, o_nlbfgs, o_vec);
        LBFGS(iter, o_y, o_s, o_rho, o_alpha, o_q, o_r, o_beta, o_ptr, o_nlbfgs, o_vec);
        extract_LBFGS_PSV(iter, G, Gp, Gu, Gpu, Gr, Gpr, P, U, R, o_r);
    } else {
        descent(G, Gp);
        descent(Gu, Gpu);
        descent(Gr, Gpr);
        store_PCG_PSV(o_new, Gp, Gpu, Gpr);
        PCG(o_new, o_old, o_dir, 3);
        extract_PCG_PSV(o_dir, G, Gu, Gr);
        store_PCG_PSV(o_old, Gp, Gpu, Gpr);
        descent(G, G);
        descent(Gu, Gu);
        descent(Gr, Gr);
    }
    grad_out(nx, ny, G, gvp);
    grad_out(nx, ny, Gu, gvs);
    grad_out(nx, ny, Gr, grho);
    float **ms[6] = {P, U, R, Gp, Gpu, Gpr};   /* grad_out freed G, Gu, Gr */
    for (int k = 0; k < 6; k++) free_matrix(ms[k], -REFH_PAD, ny + REFH_PAD, -REFH_PAD, nx + REFH_PAD);
    return o_ptr;
}
