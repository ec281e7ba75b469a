/*
 * Host file I/O of the P-SV path: .inp parameters, model files, source and
 * receiver tables, SU seismograms.  Each reader reproduces the reference's
 * reading semantics (cited per function) so that a parameter file and its data
 * files mean the same thing to both programs; rounding follows the reference's
 * float/double promotions (this file is compiled with -ffp-contract=off).
 */
#include <math.h>
#include <stddef.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "denise_b200_io.h"

int dn_fail(int code, const char *fmt, ...);

/* fd.h:17 iround(x) = (int)floor(x + 0.5), the argument promoted to double */
static int iround_d(double x) { return (int)floor(x + 0.5); }

/* ---------------------------------------------------------------------------
 * .inp reader (read_par.c:92-446)
 * ------------------------------------------------------------------------- */
enum { K_INT, K_FLT, K_STR, K_INT_NL, K_FL_LIST, K_FLT2, K_INT3, K_INT4 };

typedef struct {
    int line, kind;
    size_t off;
} line_spec;

#define OFF(f) offsetof(dn_inp, f)
/* the parameter lines of read_par.c (cases 1-115), each scanned with its own
 * format; lines past 115 are counted but not scanned, as in the reference */
static const line_spec SPEC[] = {
    {1, K_INT, OFF(mode)}, {2, K_INT, OFF(physics)}, {3, K_INT, OFF(nprocx)}, {4, K_INT, OFF(nprocy)},
    {5, K_INT, OFF(fdorder)}, {6, K_INT, OFF(maxrelerror)}, {7, K_INT, OFF(nx)}, {8, K_INT, OFF(ny)},
    {9, K_FLT, OFF(dh)}, {10, K_FLT, OFF(time)}, {11, K_FLT, OFF(dt)}, {12, K_INT, OFF(quellart)},
    {13, K_STR, OFF(signal_file)}, {14, K_FLT, OFF(ts)}, {15, K_INT, OFF(srcrec)}, {16, K_STR, OFF(source_file)},
    {17, K_INT_NL, OFF(run_multiple_shots)}, {18, K_FLT, OFF(fc_spike_1)}, {19, K_FLT, OFF(fc_spike_2)},
    {20, K_INT, OFF(order_spike)}, {21, K_INT, OFF(write_stf)}, {22, K_INT, OFF(readmod)}, {23, K_STR, OFF(mfile)},
    {24, K_INT, OFF(writemod)}, {25, K_INT, OFF(L)}, {26, K_FL_LIST, OFF(fl)}, {27, K_FLT, OFF(tau)},
    {28, K_INT, OFF(free_surf)}, {29, K_INT, OFF(fw)}, {30, K_FLT, OFF(damping)}, {31, K_FLT, OFF(fpml)},
    {32, K_FLT, OFF(npower)}, {33, K_FLT, OFF(k_max_pml)}, {34, K_INT, OFF(boundary)}, {35, K_INT, OFF(snap)},
    {36, K_INT, OFF(snap_shot)}, {37, K_FLT, OFF(tsnap1)}, {38, K_FLT, OFF(tsnap2)}, {39, K_FLT, OFF(tsnapinc)},
    {40, K_INT, OFF(idx)}, {41, K_INT, OFF(idy)}, {42, K_INT, OFF(snap_format)}, {43, K_STR, OFF(snap_file)},
    {44, K_INT, OFF(seismo)}, {45, K_INT, OFF(readrec)}, {46, K_STR, OFF(rec_file)}, {47, K_FLT2, OFF(refrec)},
    {48, K_INT, OFF(n_streamer)}, {49, K_FLT, OFF(rec_incr_x)}, {50, K_FLT, OFF(rec_incr_y)}, {51, K_INT, OFF(ndt)},
    {52, K_INT, OFF(seis_format)}, {53, K_STR, OFF(seis_file_vx)}, {54, K_STR, OFF(seis_file_vy)},
    {55, K_STR, OFF(seis_file_curl)}, {56, K_STR, OFF(seis_file_div)}, {57, K_STR, OFF(seis_file_p)},
    {58, K_STR, OFF(log_file)}, {59, K_INT, OFF(log)}, {60, K_INT, OFF(itermax)}, {61, K_STR, OFF(jacobian)},
    {62, K_STR, OFF(data_dir)}, {63, K_INT, OFF(taper)}, {64, K_INT, OFF(taperlength)}, {65, K_INT4, OFF(gradt)},
    {66, K_INT, OFF(invmat1)}, {67, K_INT, OFF(grad_form)}, {68, K_INT, OFF(quelltypb)}, {69, K_INT3, OFF(testshot)},
    {70, K_INT, OFF(sws_taper_grad_vert)}, {71, K_INT, OFF(sws_taper_grad_hor)}, {72, K_FLT, OFF(exp_taper_grad_hor)},
    {73, K_INT, OFF(sws_taper_grad_sources)}, {74, K_INT, OFF(sws_taper_circular_per_shot)},
    {75, K_INT, OFF(srtshape)}, {76, K_FLT, OFF(srtradius)}, {77, K_INT, OFF(filtsize)},
    {78, K_INT, OFF(sws_taper_file)}, {79, K_STR, OFF(tfile)}, {80, K_INT, OFF(inv_mod_out)},
    {81, K_STR, OFF(inv_modelfile)}, {82, K_FLT, OFF(vpupperlim)}, {83, K_FLT, OFF(vplowerlim)},
    {84, K_FLT, OFF(vsupperlim)}, {85, K_FLT, OFF(vslowerlim)}, {86, K_FLT, OFF(rhoupperlim)},
    {87, K_FLT, OFF(rholowerlim)}, {88, K_FLT, OFF(qsupperlim)}, {89, K_FLT, OFF(qslowerlim)},
    {90, K_INT, OFF(grad_method)}, {91, K_INT, OFF(pcg_beta)}, {92, K_INT, OFF(nlbfgs)},
    {93, K_INT, OFF(model_filter)}, {94, K_INT, OFF(filt_size)}, {95, K_INT, OFF(dtinv)},
    {96, K_FLT, OFF(eps_scale)}, {97, K_INT, OFF(stepmax)}, {98, K_FLT, OFF(scalefac)}, {99, K_INT, OFF(trkill)},
    {100, K_STR, OFF(trkill_file)}, {101, K_STR, OFF(picks_file)}, {102, K_STR, OFF(misfit_log_file)},
    {103, K_INT, OFF(min_iter)}, {104, K_INT, OFF(grad_filter)}, {105, K_INT, OFF(filt_size_grad)},
    {106, K_INT, OFF(timelapse)}, {107, K_STR, OFF(data_dir_t0)}, {108, K_INT, OFF(rtmod)},
    {109, K_INT, OFF(gravity)}, {110, K_INT, OFF(ngravb)}, {111, K_INT, OFF(nzgrav)}, {112, K_INT, OFF(grav_type)},
    {113, K_INT, OFF(back_density)}, {114, K_STR, OFF(dfile)}, {115, K_INT, OFF(rtm_shot)},
};

static void scan_line(FILE *fp, int line, dn_inp *in)
{
    static char key[4096];
    int kind = -1;
    void *dst = NULL;
    for (size_t k = 0; k < sizeof(SPEC) / sizeof(SPEC[0]); k++)
        if (SPEC[k].line == line) {
            kind = SPEC[k].kind;
            dst = (char *)in + SPEC[k].off;
        }
    if (kind < 0) return;   /* past line 115: the reference's default, no scan */
    switch (kind) {
    case K_INT: (void)!fscanf(fp, "%4095s =%i", key, (int *)dst); break;
    case K_INT_NL: (void)!fscanf(fp, "\n%4095s =%i", key, (int *)dst); break;
    case K_FLT: (void)!fscanf(fp, "%4095s =%f", key, (float *)dst); break;
    case K_STR: (void)!fscanf(fp, "%4095s =%255s", key, (char *)dst); break;
    case K_FLT2: {
        float *r = (float *)dst;   /* REFREC[1], REFREC[2] */
        (void)!fscanf(fp, "%4095s =%f ,%f", key, &r[1], &r[2]);
        break;
    }
    case K_INT3: {
        int *r = (int *)dst;       /* TESTSHOT_START, _END, _INCR */
        (void)!fscanf(fp, "%4095s =%i, %i, %i", key, &r[1], &r[2], &r[3]);
        break;
    }
    case K_INT4: {
        int *r = (int *)dst;       /* GRADT1..4 */
        (void)!fscanf(fp, "%4095s =%i, %i, %i, %i", key, &r[1], &r[2], &r[3], &r[4]);
        break;
    }
    case K_FL_LIST: {
        /* FL[1] after the key, then FL[2..L] as further numbers (L from line 25) */
        float *fl = (float *)dst, extra;
        (void)!fscanf(fp, "%4095s =%f", key, &fl[1]);
        for (int l = 2; l <= in->L; l++) (void)!fscanf(fp, "%f", l <= DN_MAX_L ? &fl[l] : &extra);
        break;
    }
    }
}

int dn_inp_read(const char *path, dn_inp *out)
{
    if (!path || !out) return dn_fail(DN_EINVAL, "dn_inp_read: null argument");
    FILE *fp = fopen(path, "r");
    if (!fp) return dn_fail(DN_EIO, "dn_inp_read: cannot open %s", path);
    memset(out, 0, sizeof(*out));
    int c, line = 0;
    while ((c = getc(fp)) != EOF) {
        /* a newline followed by anything but '#' starts a parameter line; the
         * character after the newline is consumed by the test */
        if (c == '\n' && getc(fp) != '#') {
            line++;
            scan_line(fp, line, out);
        }
    }
    fclose(fp);
    if (out->fw < 0) out->fw = 0;   /* read_par.c case 29 */
    out->lines = line;
    return DN_OK;
}

int dn_inp_nt(const dn_inp *in)
{
    const float q = in->time / in->dt;   /* float quotient, then iround */
    return iround_d(q);
}

int dn_inp_params(const dn_inp *in, float ts, dn_params *p)
{
    if (!in || !p) return dn_fail(DN_EINVAL, "dn_inp_params: null argument");
    memset(p, 0, sizeof(*p));
    p->nx = in->nx;
    p->ny = in->ny;
    p->dh = in->dh;
    p->dt = in->dt;
    p->nt = dn_inp_nt(in);
    p->fdorder = in->fdorder;
    p->maxrelerror = in->maxrelerror;
    p->free_surf = in->free_surf;
    p->fw = in->fw;
    p->damping = in->damping;
    p->fpml = in->fpml;
    p->npower = in->npower;
    p->k_max_pml = in->k_max_pml;
    p->boundary = in->boundary;
    p->L = in->L;
    if (in->L > DN_MAX_L) return dn_fail(DN_EINVAL, "L = %d: at most %d relaxation mechanisms", in->L, DN_MAX_L);
    for (int l = 1; l <= in->L; l++) p->fl[l - 1] = in->fl[l];
    p->ts = ts;
    p->invmat1 = in->invmat1 ? in->invmat1 : 1;
    p->grad_form = in->grad_form ? in->grad_form : 1;
    p->quelltypb = in->quelltypb ? in->quelltypb : 1;
    p->seismo = in->seismo;
    p->dtinv = in->dtinv > 0 ? in->dtinv : 1;
    p->snap_precision = DN_SNAP_F32;
    p->grad_accum = DN_ACC_F32;
    p->arith = DN_ARITH_EXACT;
    return DN_OK;
}

/* ---------------------------------------------------------------------------
 * model, source and receiver files
 * ------------------------------------------------------------------------- */
int dn_read_model_file(const char *path, int nx, int ny, float *out)
{
    if (!path || !out || nx < 1 || ny < 1) return dn_fail(DN_EINVAL, "dn_read_model_file: bad arguments");
    FILE *f = fopen(path, "rb");
    if (!f) return dn_fail(DN_EIO, "could not open model file %s", path);
    const size_t n = (size_t)nx * ny;
    const size_t got = fread(out, sizeof(float), n, f);
    fclose(f);
    if (got != n) return dn_fail(DN_EIO, "model file %s holds %zu of %zu values", path, got, n);
    return DN_OK;
}

int dn_read_signal_file(const char *path, int *ns, float **samples)
{
    if (!path || !ns || !samples) return dn_fail(DN_EINVAL, "dn_read_signal_file: null argument");
    *samples = NULL;
    *ns = 0;
    FILE *f = fopen(path, "r");
    if (!f) return dn_fail(DN_EIO, " Source file %s could no be opened !", path);
    int n = 0, c;
    while ((c = fgetc(f)) != EOF)   /* rd_sour.c:18-20: one sample per newline */
        if (c == '\n') n++;
    rewind(f);
    float *v = (float *)calloc((size_t)(n > 0 ? n : 1), sizeof(float));
    if (!v) {
        fclose(f);
        return dn_fail(DN_ENOMEM, "dn_read_signal_file: out of memory");
    }
    for (int k = 0; k < n; k++)
        if (fscanf(f, "%e\n", &v[k]) != 1) break;   /* unread samples stay 0, as vector() left them */
    fclose(f);
    *ns = n;
    *samples = v;
    return DN_OK;
}

int dn_read_sources(const char *path, int *nsrc, float **srcpos, float *ts)
{
    if (!path || !nsrc || !srcpos) return dn_fail(DN_EINVAL, "dn_read_sources: null argument");
    *srcpos = NULL;
    FILE *f = fopen(path, "r");
    if (!f) return dn_fail(DN_EIO, "Source file %s could not be opened", path);
    int n = 0;
    if (fscanf(f, "%d", &n) != 1 || n < 1) {
        fclose(f);
        return dn_fail(DN_EIO, "%s: no source count on the first line", path);
    }
    float *sp = (float *)calloc((size_t)n * 8, sizeof(float));
    if (!sp) {
        fclose(f);
        return dn_fail(DN_ENOMEM, "dn_read_sources: out of memory");
    }
    char cline[256];
    rewind(f);
    (void)!fgets(cline, 255, f);   /* the count line */
    float fcmax = 0.0f;
    for (int l = 0; l < n; l++) {
        float v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        if (!fgets(cline, 255, f)) {
            free(sp);
            fclose(f);
            return dn_fail(DN_EIO, "%s: %d sources announced, %d found", path, n, l);
        }
        const int nv = sscanf(cline, "%f%f%f%f%f%f%f%f", &v[0], &v[1], &v[2], &v[3], &v[4], &v[5], &v[6], &v[7]);
        if (nv < 6) {   /* sources.c:51-62: time shift, frequency and amplitude are required */
            free(sp);
            fclose(f);
            return dn_fail(DN_EIO, "Missing parameter in SOURCE_FILE %s (source %d)", path, l + 1);
        }
        float *s = sp + (size_t)l * 8;
        s[0] = v[0];                  /* x */
        s[1] = v[2];                  /* depth: the third column */
        s[2] = 0.0f;
        s[3] = v[3];                  /* tshift */
        s[4] = v[4];                  /* fc */
        s[5] = v[5];                  /* amp */
        s[6] = nv >= 7 ? v[6] : 0.0f; /* azimuth */
        /* type: the reference leaves it unset with fewer than 8 columns; an explosive source here */
        s[7] = nv >= 8 ? v[7] : 1.0f;
        if (l == 0 || s[4] > fcmax) fcmax = s[4];
    }
    fclose(f);
    *nsrc = n;
    *srcpos = sp;
    if (ts) *ts = (float)(1.0 / fcmax);   /* sources.c:88-90 */
    return DN_OK;
}

int dn_source_cell(float x, float y, float dh, int *i, int *j)
{
    if (!i || !j || !(dh > 0.0f)) return dn_fail(DN_EINVAL, "dn_source_cell: bad arguments");
    *i = iround_d(x / dh);   /* splitsrc.c: float quotient, then iround */
    *j = iround_d(y / dh);
    return DN_OK;
}

int dn_read_receivers(const char *path, const float refrec[4], float dh, int *ntr, int **rec_i, int **rec_j)
{
    if (!path || !refrec || !ntr || !rec_i || !rec_j) return dn_fail(DN_EINVAL, "dn_read_receivers: null argument");
    *rec_i = *rec_j = NULL;
    FILE *f = fopen(path, "r");
    if (!f) return dn_fail(DN_EIO, "Receiver file %s could not be opened", path);
    int n = 0, c;
    while ((c = fgetc(f)) != EOF)   /* receiver.c:36-38: one receiver per newline */
        if (c == '\n') n++;
    rewind(f);
    int *ri = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    int *rj = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    int *rk = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    if (!ri || !rj || !rk) {
        free(ri); free(rj); free(rk);
        fclose(f);
        return dn_fail(DN_ENOMEM, "dn_read_receivers: out of memory");
    }
    for (int k = 0; k < n; k++) {
        float x, y;
        if (fscanf(f, "%f%f\n", &x, &y) != 2) {
            free(ri); free(rj); free(rk);
            fclose(f);
            return dn_fail(DN_EIO, "%s: receiver %d is not a pair of numbers", path, k + 1);
        }
        ri[k] = iround_d((x + refrec[1]) / dh);
        rj[k] = iround_d((y + refrec[2]) / dh);
        rk[k] = iround_d((0.0 + refrec[3]) / dh);   /* double literal: a double quotient */
    }
    fclose(f);
    /* receiver.c:63-83: a receiver on the grid point of an earlier one is
     * flagged with a negative x index; only positive x indices are kept */
    int flag = 0;
    for (int a = 0; a < n - 1; a++)
        for (int b = a + 1; b < n; b++)
            if (ri[a] == ri[b] && rj[a] == rj[b] && rk[a] == rk[b]) ri[b] = -(++flag);
    int m = 0;
    for (int k = 0; k < n; k++)
        if (ri[k] > 0) {
            ri[m] = ri[k];
            rj[m] = rj[k];
            m++;
        }
    free(rk);
    *ntr = m;
    *rec_i = ri;
    *rec_j = rj;
    return DN_OK;
}

/* ---------------------------------------------------------------------------
 * SU output (outseis_glob.c:33-243, SEIS_FORMAT 1) and input (inseis.c)
 * The 240-byte trace header is the SEG-Y / Seismic Unix trace header; the
 * offsets below are those of its fields.
 * ------------------------------------------------------------------------- */
static void put_i32(unsigned char *h, int off, int v) { memcpy(h + off, &v, 4); }
static void put_i16(unsigned char *h, int off, short v) { memcpy(h + off, &v, 2); }
static void put_u16(unsigned char *h, int off, unsigned short v) { memcpy(h + off, &v, 2); }
static void put_f32(unsigned char *h, int off, float v) { memcpy(h + off, &v, 4); }

enum {
    SU_TRACL = 0, SU_CDP = 20, SU_TRID = 28, SU_OFFSET = 36, SU_GELEV = 40, SU_SDEPTH = 48, SU_SWDEP = 60,
    SU_SCALEL = 68, SU_SCALCO = 70, SU_SX = 72, SU_SY = 76, SU_GX = 80, SU_GY = 84, SU_NS = 114, SU_DT = 116,
    SU_D1 = 180, SU_HDR = 240
};

int dn_write_su(const char *path, const float *section, int ntr, int nt, int ndt, float dt, float time, float dh,
                const int *rec_i, const int *rec_j, const float refrec[4], float xs, float ys)
{
    if (!path || !section || !rec_i || !rec_j || !refrec || ntr < 1 || nt < 1 || ndt < 1)
        return dn_fail(DN_EINVAL, "dn_write_su: bad arguments");
    const float xshift = 800.0f, yshift = 800.0f;   /* outseis_glob.c:20 */
    const float tq = time / dt;
    const int ntt = iround_d(tq);
    const int ns2 = ntt / ndt;                      /* iround of an int quotient */
    if ((long long)ns2 * ndt > nt) return dn_fail(DN_EINVAL, "dn_write_su: section shorter than TIME/DT");
    /* receiver spacing from the first two receivers (outseis_glob.c:37) */
    const float drec = ntr > 1 ? (rec_i[1] * dh) - (rec_i[0] * dh) : 0.0f;
    FILE *f = fopen(path, "wb");
    if (!f) return dn_fail(DN_EIO, "cannot write %s", path);
    unsigned char h[SU_HDR];
    float *buf = (float *)malloc(sizeof(float) * (size_t)(ns2 > 0 ? ns2 : 1));
    if (!buf) {
        fclose(f);
        return dn_fail(DN_ENOMEM, "dn_write_su: out of memory");
    }
    const double rad2deg = 360.0 / (2.0 * 3.141592653589793);
    const unsigned short udt = (unsigned short)iround_d(((float)ndt * dt) * 1.0e6);
    int st = DN_OK;
    for (int k = 0; k < ntr; k++) {
        const float xr = rec_i[k] * dh, yr = rec_j[k] * dh;
        const float x = xr - refrec[1], y = yr - refrec[2];
        memset(h, 0, sizeof(h));
        put_i32(h, SU_TRACL, iround_d((0.0 + refrec[3]) / dh));
        put_i32(h, SU_CDP, 100 + iround_d((fabs(xr + xs) / 2.0) / drec));
        put_i16(h, SU_TRID, 1);
        const float dxs = xs - xr, dys = ys - yr;
        put_i32(h, SU_OFFSET, iround_d(sqrt(dxs * dxs + dys * dys) * 1000.0));
        put_i32(h, SU_GELEV, iround_d(yr * 1000.0));
        put_i32(h, SU_SDEPTH, iround_d(ys * 1000.0));
        put_i32(h, SU_SWDEP, iround_d((rad2deg * atan2(x - xshift, y - yshift)) * 1000.0));
        put_i16(h, SU_SCALEL, -1000);
        put_i16(h, SU_SCALCO, -1000);
        put_i32(h, SU_SX, iround_d(xs * 1000.0));
        put_i32(h, SU_GX, iround_d(xr * 1000.0));
        put_u16(h, SU_NS, (unsigned short)ns2);
        put_u16(h, SU_DT, udt);
        put_f32(h, SU_D1, (float)((float)udt * 1.0e-6));
        put_i32(h, SU_SY, iround_d(ys * 1000.0));
        put_i32(h, SU_GY, iround_d(yr * 1000.0));
        /* samples NDT, 2 NDT, ... (1-based) of the trace */
        const float *tr = section + (size_t)k * nt;
        for (int j = 1; j <= ns2; j++) buf[j - 1] = tr[(size_t)j * ndt - 1];
        if (fwrite(h, 1, SU_HDR, f) != SU_HDR || fwrite(buf, sizeof(float), (size_t)ns2, f) != (size_t)ns2) {
            st = dn_fail(DN_EIO, "write error on %s", path);
            break;
        }
    }
    free(buf);
    if (fclose(f) != 0 && st == DN_OK) st = dn_fail(DN_EIO, "write error on %s", path);
    return st;
}

int dn_write_seis(const char *path, int format, const float *section, int ntr, int nt, int ndt, float dt, float time,
                  float dh, const int *rec_i, const int *rec_j, const float refrec[4], float xs, float ys)
{
    if (format == 1) return dn_write_su(path, section, ntr, nt, ndt, dt, time, dh, rec_i, rec_j, refrec, xs, ys);
    if (format != 2 && format != 3) return dn_fail(DN_EINVAL, "SEIS_FORMAT=%d: 1 (SU), 2 (ASCII) or 3 (binary)", format);
    if (!path || !section || ntr < 1 || nt < 1 || ndt < 1) return dn_fail(DN_EINVAL, "dn_write_seis: bad arguments");
    /* outseis_glob.c:26-33 with sws = 1 (saveseis_glob.c): ns2 = iround(NT / NDT), samples NDT, 2 NDT, ... */
    const int ntt = iround_d(time / dt);
    const int ns2 = ntt / ndt;
    if ((long long)ns2 * ndt > nt) return dn_fail(DN_EINVAL, "dn_write_seis: section shorter than TIME/DT");
    FILE *f = fopen(path, format == 3 ? "wb" : "w");
    if (!f) return dn_fail(DN_EIO, "cannot write %s", path);
    int st = DN_OK;
    for (int k = 0; k < ntr && st == DN_OK; k++) {
        const float *tr = section + (size_t)k * nt;
        for (int j = 1; j <= ns2; j++) {
            const float v = tr[(size_t)j * ndt - 1];
            /* outseis_glob.c:268-295: ASCII one value per line ("%e"), or raw native floats */
            if (format == 2 ? fprintf(f, "%e\n", v) < 0 : fwrite(&v, sizeof(float), 1, f) != 1) {
                st = dn_fail(DN_EIO, "write error on %s", path);
                break;
            }
        }
    }
    if (fclose(f) != 0 && st == DN_OK) st = dn_fail(DN_EIO, "write error on %s", path);
    return st;
}

int dn_read_su(const char *path, int ntr, int ns, float *section)
{
    if (!path || !section || ntr < 1 || ns < 1) return dn_fail(DN_EINVAL, "dn_read_su: bad arguments");
    FILE *f = fopen(path, "rb");
    if (!f) return dn_fail(DN_EIO, "cannot open data file %s", path);
    unsigned char h[SU_HDR];
    int st = DN_OK;
    for (int k = 0; k < ntr && st == DN_OK; k++) {
        if (fread(h, 1, SU_HDR, f) != SU_HDR) {
            st = dn_fail(DN_EIO, "%s: trace %d missing", path, k + 1);
            break;
        }
        unsigned short hns;
        memcpy(&hns, h + SU_NS, 2);
        if ((int)hns != ns) {
            st = dn_fail(DN_EIO, "%s: trace %d has %d samples, %d expected", path, k + 1, (int)hns, ns);
            break;
        }
        if (fread(section + (size_t)k * ns, sizeof(float), (size_t)ns, f) != (size_t)ns)
            st = dn_fail(DN_EIO, "%s: trace %d is short", path, k + 1);
    }
    fclose(f);
    return st;
}
