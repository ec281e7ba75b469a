/*
 * Forward-modelling driver: MODE 0 of the reference's FD_PSV
 * (src/PSV/FD_PSV.c:197-360) for a parameter file, on the GPU library.
 *
 * Sequence, as the reference runs it: read the parameters, the models
 * (MFILE.vp/.vs/.rho, plus .qp/.qs for L > 0), the source table (which sets
 * TS = 1 / max fc) and the receiver table; one shot per line of the source
 * table, firing that source (RUN_MULTIPLE_SHOTS = 1) or all of them; a wavelet per
 * source (wavelet.c); the shot run; the seismograms written as
 * saveseis_glob.c names them, in SEIS_FORMAT 1 (SU), 2 (ASCII) or 3 (binary);
 * receivers from REC_FILE.dat, or per shot from REC_FILE_shot_<n>.dat with
 * READREC 2 (receiver.c:32-41).  The difference is that the shots run as
 * batches through one launch sequence, as many per batch as the device's free
 * memory holds.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "denise_b200_io.h"

int dn_fail(int code, const char *fmt, ...);

typedef struct {
    int nsrc, *si, *sj, *type;
    float *azi, *sig;
    float xs, ys;    /* source position written into the SU headers (srcpos[1..2][ishot]) */
} shot_src;

static void free_src(shot_src *s)
{
    free(s->si);
    free(s->sj);
    free(s->type);
    free(s->azi);
    free(s->sig);
    memset(s, 0, sizeof(*s));
}

/* receivers of shot `ishot` (1-based): REC_FILE.dat for READREC 1, REC_FILE_shot_<ishot>.dat
 * for READREC 2 (receiver.c:32-41) */
static int read_shot_receivers(const dn_inp *in, int ishot, int *ntr, int **ri, int **rj)
{
    char rpath[2 * DN_STR + 32];
    if (in->readrec == 2)
        snprintf(rpath, sizeof(rpath), "%s_shot_%i.dat", in->rec_file, ishot);
    else
        snprintf(rpath, sizeof(rpath), "%s.dat", in->rec_file);
    return dn_read_receivers(rpath, in->refrec, in->dh, ntr, ri, rj);
}

/* sources of shot `k` (0-based) in grid indices, with their wavelets (wavelet.c;
 * QUELLART 3 reads "<SIGNAL_FILE>_shot_<k+1>.dat", 7 chirps over ts = TS, and
 * the spike of QUELLART 6 is band-limited as FD_PSV.c:324-331 does) */
static int build_sources(const dn_inp *in, const dn_params *p, const float *srcpos, int nsrc, int k, int all,
                         float ts, int device, shot_src *out)
{
    memset(out, 0, sizeof(*out));
    const int first = all ? 0 : k, count = all ? nsrc : 1;
    out->si = (int *)calloc((size_t)count, sizeof(int));
    out->sj = (int *)calloc((size_t)count, sizeof(int));
    out->type = (int *)calloc((size_t)count, sizeof(int));
    out->azi = (float *)calloc((size_t)count, sizeof(float));
    out->sig = (float *)calloc((size_t)count * p->nt, sizeof(float));
    if (!out->si || !out->sj || !out->type || !out->azi || !out->sig) {
        free_src(out);
        return dn_fail(DN_ENOMEM, "driver: out of memory");
    }
    const float *s0 = srcpos + (size_t)k * 8;
    out->xs = s0[0];
    out->ys = s0[1];
    float *file_sig = NULL;
    int file_ns = 0;
    if (in->quellart == 3) {
        char path[2 * DN_STR];
        snprintf(path, sizeof(path), "%s_shot_%i.dat", in->signal_file, k + 1);
        int st = dn_read_signal_file(path, &file_ns, &file_sig);
        if (st) {
            free_src(out);
            return st;
        }
    }
    int n = 0;
    for (int l = first; l < first + count; l++) {
        const float *s = srcpos + (size_t)l * 8;
        int i, j;
        int st = dn_source_cell(s[0], s[1], p->dh, &i, &j);
        if (st) {
            free(file_sig);
            free_src(out);
            return st;
        }
        /* one rank (splitsrc.c): a source outside the grid is not injected */
        if (i < 1 || i > p->nx || j < 1 || j > p->ny) {
            fprintf(stderr, " source %d at grid point (%d,%d) lies outside the grid: not injected\n", l + 1, i, j);
            continue;
        }
        out->si[n] = i;
        out->sj[n] = j;
        out->type[n] = (int)s[7];
        out->azi[n] = s[6];
        st = dn_wavelet_ex(in->quellart, p->nt, p->dt, s[3], s[4], s[5], 0, in->fc_spike_1, in->fc_spike_2, ts,
                           file_sig, file_ns, out->sig + (size_t)n * p->nt);
        if (st) {
            free(file_sig);
            free_src(out);
            return st;
        }
        n++;
    }
    free(file_sig);
    out->nsrc = n;
    if (in->quellart == 6 && n > 0) {
        const int st = dn_tdfilt_host(out->sig, n, p->nt, p->dt, in->order_spike, in->fc_spike_2, in->fc_spike_1, device);
        if (st) {
            free_src(out);
            return st;
        }
    }
    return DN_OK;
}

static int write_shot(const dn_inp *in, const dn_params *p, dn_shot *shot, int ishot, int ntr, const int *ri,
                      const int *rj, const shot_src *src, float *buf)
{
    /* saveseis_glob.c: SEISMO 1 vx+vy, 2 p, 3 div+curl, 4 vx+vy+p; MODE 0 names <file>.shot<n> */
    static const struct { int comp; int seismo_mask; } COMPS[] = {
        {DN_SEC_VX, (1 << 1) | (1 << 4)}, {DN_SEC_VY, (1 << 1) | (1 << 4)}, {DN_SEC_P, (1 << 2) | (1 << 4)},
        {DN_SEC_DIV, 1 << 3}, {DN_SEC_CURL, 1 << 3}};
    for (size_t c = 0; c < sizeof(COMPS) / sizeof(COMPS[0]); c++) {
        if (!(COMPS[c].seismo_mask & (1 << in->seismo))) continue;
        const char *base = COMPS[c].comp == DN_SEC_VX   ? in->seis_file_vx
                           : COMPS[c].comp == DN_SEC_VY ? in->seis_file_vy
                           : COMPS[c].comp == DN_SEC_P  ? in->seis_file_p
                           : COMPS[c].comp == DN_SEC_DIV ? in->seis_file_div
                                                         : in->seis_file_curl;
        char path[2 * DN_STR];
        snprintf(path, sizeof(path), "%s.shot%d", base, ishot);
        int st = dn_shot_get_sections(shot, COMPS[c].comp, buf);
        if (!st)
            st = dn_write_seis(path, in->seis_format, buf, ntr, p->nt, in->ndt > 0 ? in->ndt : 1, p->dt, in->time,
                               p->dh, ri, rj, in->refrec, src->xs, src->ys);
        if (st) return st;
    }
    return DN_OK;
}

int dn_forward_inp(const char *inp_path, int device)
{
    dn_inp in;
    int st = dn_inp_read(inp_path, &in);
    if (st) return st;
    if (in.physics != 1) return dn_fail(DN_ENOTSUP, "PHYSICS=%d: only 2-D P-SV (1) is built", in.physics);
    if (in.readmod != 1) return dn_fail(DN_ENOTSUP, "READMOD=%d: models are read from MFILE (READMOD=1)", in.readmod);
    if (in.srcrec != 1) return dn_fail(DN_ENOTSUP, "SRCREC=%d: sources are read from SOURCE_FILE (SRCREC=1)", in.srcrec);
    if (in.readrec != 1 && in.readrec != 2)
        return dn_fail(DN_ENOTSUP, "READREC=%d: receivers are read from REC_FILE (1) or per shot (2)", in.readrec);
    if (in.seis_format < 1 || in.seis_format > 3)
        return dn_fail(DN_EINVAL, "SEIS_FORMAT=%d: SU (1), ASCII (2) or binary (3)", in.seis_format);
    if (in.seismo < 1 || in.seismo > 4) return dn_fail(DN_EINVAL, "SEISMO=%d: nothing to record", in.seismo);

    int nsrc = 0, ntr = 0, *ri = NULL, *rj = NULL, maxtr = 0;
    int *sntr = NULL, **sri = NULL, **srj = NULL;   /* per-shot receivers (READREC 2) */
    float *srcpos = NULL, ts = in.ts;
    float *mod[5] = {NULL, NULL, NULL, NULL, NULL};
    dn_model *model = NULL;
    dn_shot **shots = NULL;
    shot_src *srcs = NULL;
    float *buf = NULL;
    int nshots = 0;

    st = dn_read_sources(in.source_file, &nsrc, &srcpos, &ts);
    if (!st && in.readrec == 1) st = read_shot_receivers(&in, 1, &ntr, &ri, &rj);
    maxtr = ntr;
    if (!st && in.readrec == 2) {
        sntr = (int *)calloc((size_t)(nsrc > 0 ? nsrc : 1), sizeof(int));
        sri = (int **)calloc((size_t)(nsrc > 0 ? nsrc : 1), sizeof(int *));
        srj = (int **)calloc((size_t)(nsrc > 0 ? nsrc : 1), sizeof(int *));
        if (!sntr || !sri || !srj) st = dn_fail(DN_ENOMEM, "driver: out of memory");
        for (int k = 0; k < nsrc && !st; k++) {
            st = read_shot_receivers(&in, k + 1, &sntr[k], &sri[k], &srj[k]);
            if (!st && sntr[k] > maxtr) maxtr = sntr[k];
        }
    }
    dn_params p;
    if (!st) st = dn_inp_params(&in, ts, &p);
    if (!st) {
        static const char *EXT[5] = {"vp", "vs", "rho", "qp", "qs"};
        const int nf = in.L > 0 ? 5 : 3;
        for (int f = 0; f < nf && !st; f++) {
            mod[f] = (float *)malloc(sizeof(float) * (size_t)p.nx * p.ny);
            if (!mod[f]) {
                st = dn_fail(DN_ENOMEM, "driver: out of memory");
                break;
            }
            char mpath[2 * DN_STR];
            snprintf(mpath, sizeof(mpath), "%s.%s", in.mfile, EXT[f]);
            st = dn_read_model_file(mpath, p.nx, p.ny, mod[f]);
        }
    }
    if (!st) st = dn_model_create(&p, mod[0], mod[1], mod[2], mod[3], mod[4], device, &model);
    if (!st) {
        /* one shot per source line either way (count_src.c NSHOTS); with
         * RUN_MULTIPLE_SHOTS = 0 each of them fires all sources */
        nshots = nsrc;
        shots = (dn_shot **)calloc((size_t)nshots, sizeof(dn_shot *));
        srcs = (shot_src *)calloc((size_t)nshots, sizeof(shot_src));
        buf = (float *)malloc(sizeof(float) * (size_t)(maxtr > 0 ? maxtr : 1) * p.nt);
        if (!shots || !srcs || !buf) st = dn_fail(DN_ENOMEM, "driver: out of memory");
    }
    /* shots per batch: what the free device memory holds */
    int per_batch = nshots;
    if (!st) {
        size_t fp = 0, free_b = 0, total_b = 0;
        if (dn_shot_footprint(&p, maxtr, 0, &fp) == DN_OK && dn_device_memory(device, &free_b, &total_b) == DN_OK &&
            fp > 0) {
            const size_t fit = (size_t)(0.85 * (double)free_b) / fp;
            per_batch = fit < 1 ? 1 : (fit < (size_t)nshots ? (int)fit : nshots);
        }
    }
    for (int b0 = 0; !st && b0 < nshots; b0 += per_batch) {
        const int b1 = b0 + per_batch < nshots ? b0 + per_batch : nshots;
        for (int k = b0; k < b1 && !st; k++) {
            st = build_sources(&in, &p, srcpos, nsrc, k, !in.run_multiple_shots, ts, device, &srcs[k]);
            if (st) break;
            const int kt = in.readrec == 2 ? sntr[k] : ntr;
            dn_acq a = {srcs[k].nsrc, srcs[k].si, srcs[k].sj, srcs[k].type, srcs[k].azi, srcs[k].sig, kt,
                        in.readrec == 2 ? sri[k] : ri, in.readrec == 2 ? srj[k] : rj};
            st = dn_shot_create(model, &a, &shots[k]);
        }
        if (!st) st = dn_run(shots + b0, b1 - b0, DN_MODE_FORWARD);
        for (int k = b0; k < b1 && !st; k++)
            st = in.readrec == 2 ? write_shot(&in, &p, shots[k], k + 1, sntr[k], sri[k], srj[k], &srcs[k], buf)
                                 : write_shot(&in, &p, shots[k], k + 1, ntr, ri, rj, &srcs[k], buf);
        for (int k = b0; k < b1; k++) {
            if (shots[k]) dn_shot_destroy(shots[k]);
            shots[k] = NULL;
            free_src(&srcs[k]);
        }
    }
    if (model) dn_model_destroy(model);
    for (int f = 0; f < 5; f++) free(mod[f]);
    free(srcpos);
    free(ri);
    free(rj);
    for (int k = 0; sri && k < nsrc; k++) {
        free(sri[k]);
        free(srj[k]);
    }
    free(sntr);
    free(sri);
    free(srj);
    free(shots);
    free(srcs);
    free(buf);
    return st;
}
